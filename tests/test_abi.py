"""CPU checks of the C-ABI library: it loads, exports every entry point the
header declares, agrees with the ctypes mirror on struct layout, and rejects
bad parameters before touching the GPU."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from smectic3d_b200 import _lib as L
from smectic3d_b200.solver import Params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "smectic_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|long long|const char\*)\s+(sh_\w+)\s*\(", src, re.M)))


def test_header_declares_what_binding_knows():
    assert set(declared_symbols()) == set(L.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_string(lib):
    assert b"sm_100a" in lib.sh_version()


def test_params_struct_layout_matches_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "smectic_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(sh_params), offsetof(sh_params, dx), offsetof(sh_params, w_mid),
         offsetof(sh_params, sub_z0), offsetof(sh_params, eps_per_replica), offsetof(sh_params, curvature),
         offsetof(sh_params, replica_block), offsetof(sh_params, pencil_tile));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    got = [int(v) for v in out]
    P = L.ShParams
    assert got == [C.sizeof(P), P.dx.offset, P.w_mid.offset, P.sub_z0.offset, P.eps_per_replica.offset,
                   P.curvature.offset, P.replica_block.offset, P.pencil_tile.offset]


def test_default_params(lib):
    p = L.ShParams()
    assert lib.sh_default_params(C.byref(p)) == L.SH_OK
    assert p.n == 128 and p.batch == 1 and p.boundary == L.SH_PERIODIC
    assert p.eps == -0.75 and p.beta == 2.0 and p.gamma == 1.0 and p.q0 == 1.0
    assert abs(p.dx - 2 * 3.141592653589793 / 8) < 1e-15 and p.dt == 0.05


@pytest.mark.parametrize(
    "field,value,code",
    [
        ("n", 48, L.SH_EUNSUPPORTED),
        ("n", 1024, L.SH_EUNSUPPORTED),
        ("batch", 0, L.SH_EINVAL),
        ("boundary", 7, L.SH_EINVAL),
        ("precision", 3, L.SH_EINVAL),
        ("scheme", 9, L.SH_EINVAL),
        ("dt", -1.0, L.SH_EINVAL),
        ("dx", 0.0, L.SH_EINVAL),
        ("l1_interval", -2, L.SH_EINVAL),
        ("pencil_tile", 12, L.SH_EINVAL),
    ],
)
def test_create_rejects_bad_params(lib, field, value, code):
    p = L.ShParams()
    lib.sh_default_params(C.byref(p))
    setattr(p, field, value)
    h = C.c_void_p()
    assert lib.sh_create(C.byref(p), C.byref(h)) == code
    assert not h.value
    assert lib.sh_last_error(None)


def test_create_rejects_advection_with_substrate(lib):
    # Neumann advection (the sine-transform Stokes velocity of morphSurfK) is built;
    # combined with the substrate wall of cosNoAdvMorph it is not
    p = L.ShParams()
    lib.sh_default_params(C.byref(p))
    p.boundary = L.SH_NEUMANN
    p.advection = 1
    p.sub_sigma = 0.5
    p.sub_z0 = 1.0
    h = C.c_void_p()
    assert lib.sh_create(C.byref(p), C.byref(h)) == L.SH_EUNSUPPORTED
    assert not h.value


@pytest.mark.parametrize("boundary,z0,code", [(L.SH_PERIODIC, 1e-4, L.SH_EUNSUPPORTED), (L.SH_NEUMANN, 0.0, L.SH_EINVAL),
                                                (L.SH_NEUMANN, -1.0, L.SH_EINVAL)])
def test_create_rejects_bad_substrate(lib, boundary, z0, code):
    # the substrate penalty (cosFFT/comet/cosNoAdvMorph.cpp:67-74) is a Neumann feature with z0 > 0
    p = L.ShParams()
    lib.sh_default_params(C.byref(p))
    p.boundary = boundary
    p.sub_sigma = 0.5
    p.sub_z0 = z0
    h = C.c_void_p()
    assert lib.sh_create(C.byref(p), C.byref(h)) == code
    assert not h.value


def test_null_arguments(lib):
    assert lib.sh_create(None, None) == L.SH_EINVAL
    assert lib.sh_destroy(None) == L.SH_EINVAL
    assert lib.sh_step(None, 1) == L.SH_EINVAL
    assert lib.sh_default_params(None) == L.SH_EINVAL


@pytest.mark.parametrize("name,args", [
    ("sh_set_psi", (None, None, 0)), ("sh_set_psi_device", (None, None)), ("sh_get_psi", (None, None, 0)),
    ("sh_get_psi_device", (None, None)), ("sh_step_async", (None, 1)), ("sh_run", (None, None, 1, None, 0)),
    ("sh_energy", (None, None)), ("sh_energy_trace", (None, None, 1, None)), ("sh_l1", (None, None, None)),
    ("sh_surface_step", (None, None, None, None, None)), ("sh_local_amplitude", (None, 4, None)),
    ("sh_adjoint", (None, None, 1, None, 1, None, None, None)), ("sh_checkpoint_save", (None, None, None)),
    ("sh_checkpoint_load", (None, None, 0)), ("sh_profile_steps", (None, 1, None, None)),
    ("sh_residency", (None, None)), ("sh_synchronize", (None,)), ("sh_kernel_launches", (None, None)),
])
def test_every_handle_entry_point_rejects_a_null_handle(lib, name, args):
    assert getattr(lib, name)(*args) == L.SH_EINVAL


def test_handle_queries_on_a_null_handle(lib):
    assert lib.sh_stream(None) is None
    assert lib.sh_steps_taken(None) == -1


def test_python_params_mapping():
    p = Params(n=64, boundary="neumann", precision="fp32", scheme="imex_euler", nonlinearity="quad_cubic",
               batch=3, eps_per_replica=(-0.9, -0.7, -0.5))
    cp, keep = p.to_c()
    assert (cp.n, cp.boundary, cp.precision, cp.scheme, cp.nonlinearity) == (64, 1, 1, 1, 1)
    assert [cp.eps_per_replica[i] for i in range(3)] == [-0.9, -0.7, -0.5]
    fn = Params.from_nw(256, 16)
    assert abs(fn.dx - 2 * 3.141592653589793 / 16) < 1e-15


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No CPU fallback: without the built library the solver cannot be used."""
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", tmp_path / "libsmectic_b200.so")
    with pytest.raises(ImportError, match="is missing"):
        L.load()


def test_pencil_tiles_are_built_at_64_and_128_only(lib):
    """Tiles other than the default exist at 64^3 and at 128^3 without clusters."""
    for n, variant in ((256, 0), (128, 2), (32, 0)):
        p = L.ShParams()
        lib.sh_default_params(C.byref(p))
        p.n, p.variant, p.pencil_tile = n, variant, 32
        h = C.c_void_p()
        assert lib.sh_create(C.byref(p), C.byref(h)) == L.SH_EUNSUPPORTED, (n, variant)
        assert not h.value
