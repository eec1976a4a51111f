"""Host threads the oracle may use (TEST INFRASTRUCTURE).

PTYCHOTOMO_ORACLE_THREADS overrides; the default is every core this process
may run on.  The CPU-baseline legs time the oracle with this many threads.
"""
import os

WORKERS = int(os.environ.get("PTYCHOTOMO_ORACLE_THREADS", "0")) or len(os.sched_getaffinity(0))
