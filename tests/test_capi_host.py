"""CPU-only checks of the C-ABI library and of the host-side mirror of the reference API.

No compute call is made here (there is no GPU): the library must load, export every
symbol include/ipg.h declares, refuse to create a context without a device, and the
Python mirror must reproduce the reference's host-side rules.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import ipg
from ipg import _lib
from conftest import ROOT


def header_symbols():
    with open(os.path.join(ROOT, "include", "ipg.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"IPG_API\s+(?:const\s+)?\w+\**\s+\**(ipg_\w+)\s*\(", text)))


def test_header_declares_api():
    syms = header_symbols()
    assert len(syms) >= 25
    assert sorted(_lib.API_SYMBOLS) == syms


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for s in header_symbols():
        assert hasattr(L, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ipg_\w+)", out))
    assert set(header_symbols()) <= exported
    # nothing but the declared API is exported
    assert exported == set(header_symbols())


def test_library_is_built_for_sm100a_only():
    """build.py compiles every kernel for sm_100a and nothing else (ipg_create also checks at
    run time that the kernels' binary version is 10.0 before it makes a context)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("ipg_build", os.path.join(ROOT, "interatomicpotentials.jl_b200",
                                                                            "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    assert b.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_no_device_is_reported():
    import ctypes as C
    if _has_gpu():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert _lib.lib().ipg_create(0, C.byref(h)) == -9
    with pytest.raises(ipg.IPGError):
        ipg.Context(0)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_version():
    assert _lib.lib().ipg_version() == 100


# ---- host mirror ------------------------------------------------------------------
def test_linear_combination_algebra():
    """test/unit/mixed/linear_combination_potential.jl: +, -, *, / build the same sums."""
    a = ipg.LennardJones(1.0, 1.0, 2.0, ["Ar"])
    b = ipg.Morse(1.0, 1.0, 1.0, 3.0, ["Ar"])
    c = ipg.Coulomb(1.0, 1.0, 4.0, ["Ar"])
    p = a + b
    assert p.potentials == [a, b] and p.coefficients == [1.0, 1.0]
    assert (a - b).coefficients == [1.0, -1.0]
    assert (2 * a).coefficients == [2.0]
    assert (a / 4).coefficients == [0.25]
    assert (-a).coefficients == [-1.0]
    assert (a + b + c).get_rcutoff() == 4.0
    assert (a + b).get_species() is None
    assert (a + (b + c)) == (a + b + c)
    assert (3 * (a + b)).coefficients == [3.0, 3.0]
    assert ipg.AbstractPotential().get_rcutoff() == np.inf


def test_species_mask():
    a = ipg.LennardJones(1.0, 1.0, 2.0, ["Ar", "Xe"])
    t = a.term({"Ar": 0, "H": 1, "Xe": 2})
    assert t.species_mask == 0b101
    t = ipg.LennardJones(1.0, 1.0, 2.0, None).term({"Ar": 0})
    assert t.species_mask == (1 << 64) - 1
    assert t.kind == 1 and t.params[0] == 1.0


def test_num_snap_coeffs():
    """utl.jl:8-25."""
    assert [ipg.get_num_snap_coeffs(J, 1, False) for J in range(9)] == [1, 2, 5, 8, 14, 20, 30, 40, 55]
    assert ipg.get_num_snap_coeffs(8, 2, True) == 55 * 8


def test_system_box():
    s = ipg.System(np.zeros((2, 3)), ["A", "B"], np.diag([1.0, 2.0, 3.0]), (True, False, True))
    assert np.array_equal(s.L, [1.0, np.inf, 3.0])
    assert s.unique_symbols() == ["A", "B"]


def test_units_codata2018():
    assert abs(ipg.units.eV * 27.211386245988 - 1.0) < 1e-15
    assert abs(ipg.units.angstrom * 0.529177210903 - 1.0) < 1e-15


def test_flop_counts_consistent():
    from ipg import flops as F
    assert F.snap_atom_kernel(8, 1, 26, "plain") > F.snap_atom_kernel(8, 1, 26, "adjoint") > 0
    assert F.z_atom(8) > F.z_atom(6)


def test_context_closes_its_snap_handles_first(monkeypatch):
    """Finalizers of a context and its SNAP objects may run in any order (a reference cycle
    collected at exit): closing the context closes the SNAP handles first, and a SNAP whose
    context is gone does not call into the library."""
    import weakref
    import ipg.context as ctxmod
    import ipg.snap as snapmod
    calls = []

    class FakeLib:
        def ipg_destroy(self, h):
            calls.append(("ctx", h))

        def ipg_snap_destroy(self, h):
            calls.append(("snap", h))

    monkeypatch.setattr(ctxmod, "lib", lambda: FakeLib())
    monkeypatch.setattr(snapmod, "lib", lambda: FakeLib())
    ctx = object.__new__(ctxmod.Context)  # no device here: only the handle bookkeeping
    ctx._h, ctx._dependents = "c", weakref.WeakSet()
    snap = object.__new__(snapmod.SNAP)
    snap._h, snap.ctx = "s", ctx
    ctx._register(snap)
    ctx.close()
    assert calls == [("snap", "s"), ("ctx", "c")]
    snap.close()  # already closed: nothing more
    ctx2 = object.__new__(ctxmod.Context)
    ctx2._h, ctx2._dependents = None, weakref.WeakSet()  # a context finalized first
    snap2 = object.__new__(snapmod.SNAP)
    snap2._h, snap2.ctx = "s2", ctx2
    snap2.close()
    assert calls == [("snap", "s"), ("ctx", "c")] and snap2._h is None
