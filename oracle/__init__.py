"""CPU oracle for the ptycho-tomography hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
package; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may use it, and only as the checker or the timed CPU
baseline.

Contents
--------
usfft   NumPy restatement of the reference USFFT Radon operator
        (src/cuda/radonusfft.cu:5-144, src/include/kernels.cuh:5-216).
ptycho  NumPy restatement of the reference ptychography operator
        (src/cuda/ptychofft.cu:5-93, src/include/kernels.cuh:243-355).
solver  NumPy restatement of src/ptychotomo/solver.py (CuPy replaced by
        NumPy, reductions in float64).
nudft   complex128 direct-sum operators that the USFFT and ptycho
        operators approximate / equal (precision study oracle).

Pinning: the restatement is checked against the reference's own CUDA
operators (compiled unmodified from the reference sources by
``oracle/Makefile`` into ``oracle/_ref``) through golden vectors stored in
``tests/golden`` and generated by ``tests/golden/make_golden.py`` on a GPU.
"""
