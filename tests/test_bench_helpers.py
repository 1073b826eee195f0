"""Host-side helpers of bench.py that shape its JSON line: the per-part solve breakdown, the
ncu launch-list summary and the peak error of eps2 (no GPU needed)."""
import math

import numpy as np

import bench


def _stats(**kw):
    st = {"tri_ms": 0.0, "hemv_ms": 0.0, "her2k_ms": 0.0, "her2k_flops": 0.0, "tdsolve_ms": 0.0}
    st.update(kw)
    return st


def test_solve_breakdown_per_step_and_rates():
    st = _stats(tri_ms=2000.0, hemv_ms=1200.0, her2k_ms=400.0, her2k_flops=8e12, tdsolve_ms=100.0)
    b = bench.solve_breakdown(st, 2)
    assert b["tridiagonalise"] == 1.0 and b["hemv"] == 0.6 and b["her2k"] == 0.2
    assert math.isclose(b["column_kernels_and_gaps"], 0.2)
    assert b["tridiagonal_solve"] == 0.05
    assert math.isclose(b["her2k_tflops"], 20.0)
    assert math.isclose(b["her2k_frac_of_nominal_fp64_40"], 0.5)
    assert bench.solve_breakdown(_stats(), 1) is None   # not profiled


def test_ncu_launch_summary_aggregates_kernels(tmp_path):
    rows = [
        '"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size",'
        '"Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"',
        '"0","1","python","h","void <unnamed>::k_hemv(CUtensorMap_st, const double2 *)","1","7","(256, 1, 1)",'
        '"(148, 1, 1)","0","10.0","Command line profiler metrics","gpu__time_duration.sum","us","100.5"',
        '"1","1","python","h","<unnamed>::k_colA(double2 *)","1","7","(256, 1, 1)","(10, 1, 1)","0","10.0",'
        '"Command line profiler metrics","gpu__time_duration.sum","ns","2,500"',
        '"2","1","python","h","void <unnamed>::k_hemv(CUtensorMap_st, const double2 *)","1","7","(256, 1, 1)",'
        '"(148, 1, 1)","0","10.0","Command line profiler metrics","gpu__time_duration.sum","us","99.5"',
    ]
    p = tmp_path / "l.csv"
    p.write_text("==PROF== noise line\n" + "\n".join(rows) + "\n")
    out = bench.ncu_launch_summary(str(p)).splitlines()
    assert out[1].split()[:3] == ["k_hemv", "2", "0.200"]
    assert out[2].split()[:3] == ["k_colA", "1", "0.003"]
    assert out[-1].split()[:3] == ["total", "3", "0.203"]


def test_peak_rel_error_reads_the_maxima():
    x = np.linspace(0, 6, 601)
    ref = np.exp(-((x - 2) / 0.1) ** 2) + 0.5 * np.exp(-((x - 4) / 0.1) ** 2)
    got = ref.copy()
    got[400] += 0.01        # at the second peak
    got[100] += 0.5         # far from any peak: not counted
    assert math.isclose(bench.peak_rel_error(ref, got), 0.01, rel_tol=1e-9)
