"""The C ABI exposed as torch.library custom ops (no GPU needed here).

Checks that every op is registered under ``torch.ops.shearwave_b200`` with
the schema the host API relies on (which arguments it writes), that the fake
implementations give the output shapes without running a kernel (what
FakeTensor tracing and ``torch.compile`` use), and that a CPU tensor is
refused by the dispatcher: there is no CPU path.
"""

from __future__ import annotations

import pytest
import torch

import shearwave_b200.ops  # noqa: F401  (registers the ops)

OPS = {
    "laplacian": set(), "divergence": set(), "gradient": set(), "project": set(),
    "project_batch": set(), "convert_": {"dst"}, "static_solve": set(), "strain": set(),
    "strain_aos": set(), "strain_invariants": set(), "arf_envelope": set(), "arf_force": set(),
    "fdtd_materials_": {"coef", "inv_rho"}, "fdtd_init_": {"state"},
    "fdtd_steps_": {"state", "snaps", "traces", "flags", "clock", "queue"},
    "fdtd_finish": {"flags"}, "fdtd_reproject_": {"state"},
    "fdtd_batch_steps_": {"state", "flags", "queue"},
}


def _schema(name):
    return getattr(torch.ops.shearwave_b200, name).default._schema


@pytest.mark.parametrize("name", sorted(OPS))
def test_registered_with_declared_writes(name):
    sch = _schema(name)
    written = {a.name for a in sch.arguments if a.alias_info is not None and a.alias_info.is_write}
    assert written == OPS[name], (name, written)


def test_cpu_tensors_are_refused():
    with pytest.raises(NotImplementedError):
        torch.ops.shearwave_b200.laplacian(torch.zeros(4, 4, 4), [1.0, 1.0, 1.0])


def test_fake_shapes():
    from torch._subclasses.fake_tensor import FakeTensorMode

    ops = torch.ops.shearwave_b200
    with FakeTensorMode():
        f = torch.empty((9, 10, 11), dtype=torch.float32, device="cuda")
        assert ops.laplacian(f, [1.0, 1.0, 1.0]).shape == f.shape
        assert ops.divergence(f, f, f, [1.0, 1.0, 1.0]).shape == f.shape
        assert all(g.shape == f.shape for g in ops.gradient(f, [1.0, 1.0, 1.0]))
        fs, st = ops.project(None, None, f, [1.0, 1.0, 1.0], 1e-6, 10, "cg")
        assert tuple(fs.shape) == (3, 9 * 10 * 16) and fs.dtype == torch.float64
        assert tuple(st.shape) == (4,) and st.device.type == "cpu"
        outs, st = ops.project_batch([None, f], [None, f], [f, f], [1.0] * 6, [1e-6] * 2, [5, 5])
        assert len(outs) == 2 and tuple(st.shape) == (2, 4)
        eps, vol, dev, ms, vm = ops.strain(f, f, f, [1.0, 1.0, 1.0], True, True)
        assert tuple(eps.shape) == (9, 10, 11, 6) and vm.dtype == torch.float64
        u = torch.empty((9, 10, 11, 3), dtype=torch.float64, device="cuda")
        eps, *inv = ops.strain_aos(u, [1.0, 1.0, 1.0], False)
        assert eps.numel() == 0 and all(tuple(t.shape) == (9, 10, 11) for t in inv)
        inv = ops.strain_invariants(torch.empty((5, 6), device="cuda"))
        assert tuple(inv[0].shape) == (5,) and inv[3].dtype == torch.float64
        u, s = ops.static_solve(f, None, 2.0, [1.0, 1.0, 1.0], 1e-6, 10)
        assert tuple(u.shape) == (1, 9 * 10 * 16)


def test_host_api_computes_through_the_ops_only():
    """Every compute entry point of the C ABI is reached through torch.ops:
    the host modules call the ctypes binding directly only for the device
    selection and the launch-shape knobs."""
    import re

    from conftest import ROOT

    allowed = {"sw_set_device", "sw_tune_set"}
    for mod in ("solver", "strain", "radiation", "serve", "validation", "tune", "_device"):
        text = (ROOT / "shearwave_b200" / f"{mod}.py").read_text()
        called = set(re.findall(r"""\.call\(\s*["'](sw_[a-z0-9_]+)["']""", text))
        assert called <= allowed, (mod, called - allowed)
