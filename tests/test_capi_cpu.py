"""The C ABI without a GPU: the library loads, exports every entry point that
include/m3lb.h declares, and rejects invalid arguments before touching CUDA."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from m3lb_b200 import capi
from m3lb_b200 import solver as S


def declared():
    text = capi.HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(m3lb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (m3lb_[a-z0-9_]+)", out))
    assert set(names) == exported, (set(names) ^ exported)
    # the Python binding covers all of them
    assert set(names) == set(capi.SIGNATURES)


@pytest.mark.parametrize("args,code,msg", [
    ((5, 8, 8, 8, 1, 1, 1, 4, 0, 1, 1, 0), capi.ERR_INVALID, "lattice"),
    ((27, 0, 8, 8, 1, 1, 1, 4, 0, 1, 1, 0), capi.ERR_INVALID, "extents"),
    ((9, 8, 8, 2, 1, 1, 1, 1, 0, 0, 1, 0), capi.ERR_INVALID, "D2Q9"),
    ((27, 8, 8, 8, 1, 1, 1, 7, 0, 0, 1, 0), capi.ERR_INVALID, "operator"),
    ((27, 8, 8, 8, 1, 1, 1, 1, 3, 0, 1, 0), capi.ERR_INVALID, "equilibrium"),
    ((27, 8, 8, 8, 1, 1, 1, 1, 0, 9, 1, 0), capi.ERR_INVALID, "storage"),
    ((27, 8, 8, 8, 1, 1, 1, 4, 0, 1, 0, 0), capi.ERR_UNSUPPORTED, "16-bit"),
    ((27, 2000, 2000, 2000, 1, 1, 1, 4, 0, 1, 1, 0), capi.ERR_INVALID, "2^31"),
])
def test_create_rejects_bad_arguments(args, code, msg):
    h = C.c_void_p()
    rc = capi.lib().m3lb_create(*args, C.byref(h))
    assert rc == code
    assert msg in capi.last_error()
    assert not h.value


def test_null_handles_are_errors_not_crashes():
    lib = capi.lib()
    assert lib.m3lb_step(None, 1, 0) == capi.ERR_INVALID
    assert lib.m3lb_destroy(None) == capi.OK
    assert lib.m3lb_reduce(None, None) == capi.ERR_INVALID
    assert lib.m3lb_gather(None, None) == capi.ERR_INVALID


def test_footprint_budget():
    # 256^3 D3Q27 FP16: 27 * 2 B per node of populations, 1 B flags, 16 B fields
    b = capi.footprint(27, 256, 256, 256, storage=capi.STORE_F16)
    n = 256 ** 3
    assert n * (54 + 1 + 16) <= b <= n * (54 + 1 + 16) * 1.01
    b32 = capi.footprint(27, 256, 256, 256, storage=capi.STORE_F32)
    assert b32 > b
    # halo rows count in non-periodic directions
    assert capi.footprint(9, 64, 32, 1, True, False, True) > capi.footprint(9, 64, 32, 1)


@pytest.mark.parametrize("shape,per", [((8, 6, 1), (True, True, True)),
                                       ((8, 6, 5), (True, False, True)),
                                       ((7, 6, 5), (False, False, False)),
                                       ((9, 1, 1), (False, False, False))])
def test_domain_mirror_matches_reference_geometry(shape, per):
    """Domain.hpp:47-56, 104-108: halo only on non-periodic axes with n > 1."""
    import oracle as O
    d = S.Domain(*shape, *per)
    o = O.CpuSolver("oracle", lattice=27 if shape[2] > 1 else 9, op="none", nx=shape[0],
                    ny=shape[1], nz=shape[2], px=per[0], py=per[1], pz=per[2])
    assert d.n_padded == o.n_padded
    x, y, z = 1, 0, 0
    assert d.coords(d.id(x, y, z)) == (x + d.hx, y + d.hy, z + d.hz)


def test_policy_mirror_defaults():
    """Defaults and helpers of the reference's policies (BGK.hpp:43-52,
    TRT.hpp:46-62, MomentCollision.hpp:89-101)."""
    b = S.BGK()
    assert b.storage is S.RawPopulations and not b.forcing.active
    assert b.omega_from_viscosity(b.viscosity_from_omega(1.3)) == pytest.approx(1.3)
    t = S.TRT()
    wm = t.omega_minus_for(1.25, t.magic_3_16)
    assert t.magic_parameter(1.25, wm) == pytest.approx(3 / 16)
    cm = S.CentralMoments()
    assert cm.op == capi.OP_CM and cm.bulk() == cm.omega
    assert S.MRT().op == capi.OP_MRT
    assert [S.opp(i) for i in range(5)] == [0, 2, 1, 4, 3]
    for L in (S.D2Q9, S.D3Q27):
        assert sum(L.w) == pytest.approx(1.0)
        for i in range(L.Q):
            j = S.opp(i)
            assert (L.cx[j], L.cy[j], L.cz[j]) == (-L.cx[i], -L.cy[i], -L.cz[i])


def test_scalar_create_checks_extents_before_device_work():
    # the scalar kernels take y and z from the grid, so ny and nz are at most 65535
    lib = capi.lib()
    h = C.c_void_p()
    bgk = 1  # M3LB_SOP_BGK
    assert lib.m3lb_scalar_create(7, 4, 70000, 2, 1, 1, 1, bgk, capi.STORE_F32, C.byref(h)) == \
        capi.ERR_INVALID
    assert "65535" in capi.last_error()
    assert lib.m3lb_scalar_create(7, 4, 4, 4, 1, 1, 1, 2, capi.STORE_F16, C.byref(h)) == \
        capi.ERR_UNSUPPORTED
    assert not h.value


def test_noalloc_scratch_address_is_kept_per_context(tmp_path):
    """m3lb_reduce_static's scratch address is cached per CUDA context, not
    per device: the cache logic (ctx_cache.h) compiled on the host looks an
    address up again when the context ID changes (as after cudaDeviceReset)
    and never keeps one looked up under an unknown context."""
    import shutil
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    exe = tmp_path / "ctx_cache_case"
    cxx = shutil.which("g++") or "g++"
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Werror",
                        f"-I{root / 'm3lb_b200' / 'csrc'}",
                        str(root / "tests" / "cpp" / "ctx_cache_case.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
