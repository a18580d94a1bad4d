"""The runner's GPU timeline summary (busy fraction, idle gaps between device activities) on a
hand-made trace."""
from dac_vtsa_b200.runner import timeline_summary


def test_timeline_summary_counts_busy_time_and_gaps():
    ev = [
        {"cat": "kernel", "name": "void dv::k_setup(int)", "ts": 0.0, "dur": 5.0},          # before the first sweep
        {"cat": "kernel", "name": "void dv::k_pc_apply<7, 3, double, true>(PcGeom)", "ts": 100.0, "dur": 40.0},
        {"cat": "kernel", "name": "void dv::k_cprops<2>(int)", "ts": 142.0, "dur": 8.0},    # 2 us gap: not listed
        {"cat": "kernel", "name": "dv::k_cgs_orth_norm(long)", "ts": 150.0, "dur": 10.0},
        {"cat": "kernel", "name": "void dv::k_pc_apply<7, 3, double, true>(PcGeom)", "ts": 180.0, "dur": 40.0},
        {"cat": "gpu_memcpy", "name": "Memcpy DtoH (Device -> Pinned)", "ts": 230.0, "dur": 2.0},
        {"cat": "cuda_runtime", "name": "cudaStreamSynchronize", "ts": 225.0, "dur": 9.0},
    ]
    s = timeline_summary(ev)
    assert s["span_us"] == 132.0
    assert s["kernel_us"] == 98.0
    assert abs(s["busy_fraction"] - 98.0 / 132.0) < 1e-12
    gaps = {g["between"]: (g["count"], g["total_us"]) for g in s["idle_gaps_over_5us"]}
    assert gaps == {"k_cgs_orth_norm -> k_pc_apply<7, 3, double, true>": (1, 20),
                    "k_pc_apply<7, 3, double, true> -> gpu_memcpy:Memcpy DtoH": (1, 10)}
    k = {r["kernel"]: (r["count"], r["total_us"]) for r in s["kernels"]}
    assert k["k_pc_apply<7, 3, double, true>"] == (2, 80)
    assert "k_setup" not in k
