"""bench.py's byte model and roofline bookkeeping (CPU): the pass-model
bytes per operator, the DRAM traffic figure only for a captured split and
workload, and the workload description."""
import bench


def test_pass_model_bytes():
    c = dict(bench.CFG)
    b = bench.workload_bytes(c)
    n, nz, nt = c["n"], c["nz"], c["ntheta"]
    G = 3 * n
    assert b["radon_fwd"] == b["radon_adj"] == 8 * nz * (n * n + 4 * G * G + nt * n)
    S = nt * c["nside"] ** 2
    assert b["ptycho_fwd"] == b["ptycho_adj"] == 8 * S * (c["nprb"] ** 2 + c["det"] ** 2)
    assert abs(b["radon_fwd"] / 1e9 - 5.167) < 1e-3 and abs(b["ptycho_adj"] / 1e9 - 17.012) < 1e-3


def test_dram_traffic_only_where_captured():
    c = dict(bench.CFG)
    frames = c["ntheta"] * c["nside"] ** 2
    for parts, per_frame in bench.PTYCHO_ADJ128_DRAM_PER_FRAME.items():
        assert bench.dram_traffic(c, parts) == int(round(per_frame * frames))
        assert "parts %d" % parts in bench.traffic_source(parts)
    assert bench.dram_traffic(c, 2) is None                      # no capture for this split
    assert bench.dram_traffic(dict(c, ntheta=96), 1) is None     # fewer angles than SMs
    assert bench.dram_traffic(dict(c, det=64, nprb=64), 1) is None


def test_config_names_the_workload():
    d = bench.config_dict(dict(bench.CFG), {"autotuned": {"radon_gather": bench.GATHER_NAMES[2]}})
    assert d["workload"].startswith("radonusfft fwd+adj (n=nz=256, 384 angles, M=7)")
    assert d["autotuned"]["radon_gather"] == "TMA smem tiles"
    assert "L2" not in d["workload"] and "no flush" in d["l2"]
