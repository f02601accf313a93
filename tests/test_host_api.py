"""Host-side argument handling of the drop-in API (no GPU needed).

Every check below raises before the first device call, with the reference's
messages (src/shearwave/solver.py:88-171, 287-308, 396-408, 1060-1079;
src/shearwave/strain.py:98-100, 138-159).
"""

from __future__ import annotations

import numpy as np
import pytest

import shearwave_b200 as sw

Z = np.zeros((6, 5, 4), np.float32)


def _call(**kw):
    args = dict(bx=None, by=None, bz=Z, rho=1000.0, mu=2000.0, dX=1e-3, dY=1e-3, dZ=1e-3,
                dT=1e-6, n_steps=4, opts=None)
    args.update(kw)
    return sw.shear_fdtd(**args)


def test_requires_a_force_component():
    with pytest.raises(ValueError, match="At least one body-force component"):
        _call(bz=None)


def test_negative_reproject_every():
    with pytest.raises(ValueError, match="reproject_every"):
        _call(opts={"env_t": np.ones(4), "reproject_every": -1})


def test_env_t_length():
    with pytest.raises(ValueError, match=r"env_t length \(3\) must equal n_steps \(4\)"):
        _call(opts={"env_t": np.ones(3)})


def test_body_force_shape():
    with pytest.raises(ValueError, match="Body-force component has incompatible shape"):
        _call(bx=np.zeros((6, 5, 3), np.float32))
    with pytest.raises(ValueError, match="Body-force component has incompatible shape"):
        _call(bz=np.zeros((6, 5, 4, 3), np.float32))


def test_material_shape():
    with pytest.raises(ValueError, match="Material field has incompatible shape"):
        _call(rho=np.ones((6, 5, 3)))
    with pytest.raises(ValueError, match="Material field has incompatible shape"):
        _call(opts={"eta": np.ones((2, 2, 2))})


def test_initial_state_shape():
    with pytest.raises(ValueError, match=r"initial_u must match shape"):
        _call(opts={"initial_u": np.zeros((6, 5, 4))})
    with pytest.raises(ValueError, match=r"initial_v must match shape"):
        _call(opts={"initial_v": np.zeros((6, 5, 4, 2))})


def test_snapshot_stride_errors():
    with pytest.raises(ValueError, match="positive integer"):
        _call(snapshot_stride=0)
    with pytest.raises(ValueError, match="multiple of snapshot_stride"):
        _call(snapshot_stride=3)
    with pytest.raises(ValueError, match="not both supported"):
        _call(snapshot_stride=2, return_traces=True, trace_indices=([0], [0], [0]))


def test_trace_errors():
    with pytest.raises(ValueError, match="trace_indices must be provided"):
        _call(return_traces=True)
    with pytest.raises(ValueError, match="3-tuple"):
        _call(trace_indices=([0], [0]))
    with pytest.raises(ValueError, match="same shape"):
        _call(trace_indices=([0], [0, 1], [0]))
    with pytest.raises(ValueError, match="1D"):
        _call(trace_indices=([[0]], [[0]], [[0]]))
    with pytest.raises(ValueError, match="outside the grid"):
        _call(trace_indices=([6], [0], [0]), return_traces=True)


def test_jax_entry_point_errors():
    with pytest.raises(ValueError, match="callback is not supported"):
        sw.shear_fdtd_jax(None, None, Z, 1000.0, 2000.0, 1e-3, 1e-3, 1e-3, 1e-6, 4,
                          callback=lambda it, u: None)
    with pytest.raises(NotImplementedError, match="reproject_every"):
        sw.shear_fdtd_jax(None, None, Z, 1000.0, 2000.0, 1e-3, 1e-3, 1e-3, 1e-6, 4,
                          opts={"reproject_every": 5})


def test_unknown_precision():
    with pytest.raises(ValueError, match="precision"):
        _call(opts={"precision": "bf16"})


def test_strain_validation():
    with pytest.raises(ValueError, match="same shape"):
        sw.compute_strain_tensor(np.zeros((4, 4, 4)), np.zeros((4, 4, 5)), np.zeros((4, 4, 4)),
                                 1e-3, 1e-3, 1e-3)
    with pytest.raises(ValueError, match="positive"):
        sw.compute_strain_tensor(Z, Z, Z, -1e-3, 1e-3, 1e-3)
    with pytest.raises(ValueError, match="3-D"):
        sw.compute_strain_tensor(np.zeros((4, 4)), np.zeros((4, 4)), np.zeros((4, 4)),
                                 1e-3, 1e-3, 1e-3)
    with pytest.raises(ValueError, match="Voigt"):
        sw.compute_strain_invariants(np.zeros((5, 5, 5, 3)))


def test_no_cpu_fallback_without_a_gpu():
    """With valid arguments and no CUDA device the call fails loudly."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        _call(opts={"env_t": np.ones(4)})


def test_hann1d_matches_reference_definition():
    """hann1d (solver.py:1053-1057): numpy's Hann window as float32, ones for n <= 1."""
    import numpy as np

    from shearwave_b200 import hann1d

    assert hann1d(0).shape == (0,) and hann1d(1).tolist() == [1.0]
    w = hann1d(9)
    assert w.dtype == np.float32
    assert np.array_equal(w, np.hanning(9).astype(np.float32))


def test_arrival_analysis_recovers_a_known_speed():
    """Synthetic traces with pulses arriving at distance / c: the fit returns c."""
    import numpy as np

    from shearwave_b200.validation import arrival_analysis

    dT, c = 1e-5, 2.5
    dist = np.array([3e-3, 5e-3, 7e-3, 9e-3])
    t = np.arange(800) * dT
    traces = np.stack([np.tanh((t - d / c) / 4e-5) for d in dist])  # velocity peaks at d/c
    r = arrival_analysis(traces, dT, dist, c)
    assert abs(r["c_fit"] - c) / c < 0.02
    assert np.all(np.abs(r["speeds"] - c) / c < 0.05)


def test_bench_traffic_table_covers_both_step_kernels():
    """bench.py's roofline reads the ncu bytes per cell-step of whichever step
    kernel the run used from profiles/traffic.txt: both must be there, and
    the two-step kernel must move fewer bytes than the one-step kernel."""
    import importlib.util
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    spec = importlib.util.spec_from_file_location("bench_for_test", root / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    one = bench.ncu_bytes_per_cell_step("step_f32_tma")
    two = bench.ncu_bytes_per_cell_step("step_f32_fused2")
    assert one is not None and two is not None
    assert 0 < two < one
    assert bench.ncu_bytes_per_cell_step("no_such_kernel") is None


def _load_bench():
    import importlib.util
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    spec = importlib.util.spec_from_file_location("bench_for_test", root / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_serving_request_pool_is_seeded_and_bounded(monkeypatch):
    """A long config-4 stream draws its arrivals from a small pool of
    distinct seeded requests: the same order for the same seed, every entry
    one of the pool's objects (nothing regenerated per arrival)."""
    bench = _load_bench()
    from shearwave_b200 import workloads as W

    made = []

    def fake_c4(rng):  # the generator's draws without building grids
        made.append(int(rng.integers(0, 1 << 30)))
        return {"id": made[-1]}

    monkeypatch.setattr(W, "problem_c4", fake_c4)
    a = bench.c4_requests(500, seed=3, pool=8)
    b = bench.c4_requests(500, seed=3, pool=8)
    assert len(a) == 500 and len({id(p) for p in a}) <= 8
    assert [p["id"] for p in a] == [p["id"] for p in b]
    assert len(made) == 16  # 8 per call
    full = bench.c4_requests(20, seed=3, pool=0)
    assert len({id(p) for p in full}) == 20


def test_clock_sampler_without_nvidia_smi_reports_unavailable(monkeypatch):
    """The bench's clock sampler starts before the timed region; with no
    nvidia-smi (as on a CPU-only machine) it reports no samples instead of
    failing the run."""
    bench = _load_bench()

    def no_smi(*a, **k):
        raise FileNotFoundError("nvidia-smi")

    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    with bench.ClockSampler(0) as c:
        pass
    assert c.summary()["samples"] == 0
