"""CPU-side checks of the product boundary (no GPU compute here).

- libgranite_ccz4.so builds for sm_100a and loads, and exports every function
  that include/granite_ccz4.h declares;
- the header compiles as C and C++;
- without a GPU the library reports GRANITE_ERR_NO_DEVICE instead of crashing
  or falling back to a CPU path;
- host-side logic (GridBlock layout and coordinates, initial data) matches the
  oracle's conventions.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import Geom

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "granite_ccz4.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(granite_ccz4_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from granite_b200 import build
    path = build.build()
    return C.CDLL(path)


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ["granite_ccz4_create", "granite_ccz4_destroy", "granite_ccz4_compute_rhs_host",
              "granite_ccz4_apply_dissipation_host", "granite_ccz4_compute_constraints_host",
              "granite_ccz4_rk3_step", "granite_ccz4_hierarchy_step",
              "granite_ccz4_constraint_norms", "granite_ccz4_last_error"]:
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_exports_nothing_else():
    from granite_b200 import build
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    ours = {e for e in exported if e.startswith("granite_")}
    assert ours == set(declared_functions())


@pytest.mark.parametrize("compiler,flag", [("/usr/bin/gcc", "-std=c99"), ("/usr/bin/g++", "-std=c++17")])
def test_header_compiles(tmp_path, compiler, flag):
    if not os.path.exists(compiler):
        pytest.skip("no system compiler")
    src = tmp_path / ("t.c" if "gcc" in compiler else "t.cpp")
    src.write_text('#include "granite_ccz4.h"\nint main(void){granite_ccz4_params p;'
                   'granite_ccz4_default_params(&p);return p.fd_order == 4 ? 0 : 1;}\n')
    subprocess.run([compiler, flag, "-Wall", "-Werror", "-c", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(tmp_path / "t.o")], check=True)


def test_abi_version_and_defaults(lib):
    assert lib.granite_ccz4_abi_version() == 1
    import granite_b200 as gb
    p = gb._Params()
    lib.granite_ccz4_default_params(C.byref(p))
    assert (p.kappa1, p.kappa2, p.eta, p.ko_sigma) == (0.02, 0.0, 2.0, 0.1)
    assert (p.chi_blend_center, p.chi_blend_width, p.fd_order) == (0.05, 0.02, 4)


def test_no_device_is_an_error_not_a_fallback(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    import granite_b200 as gb
    p = gb._Params()
    lib.granite_ccz4_default_params(C.byref(p))
    h = C.c_void_p()
    rc = lib.granite_ccz4_create(C.byref(p), C.byref(h))
    assert rc == -3 and not h.value
    with pytest.raises(gb.GraniteError):
        gb.CCZ4Evolution(gb.CCZ4Params())


def test_invalid_arguments_rejected(lib):
    import granite_b200 as gb
    p = gb._Params()
    lib.granite_ccz4_default_params(C.byref(p))
    p.fd_order = 6
    h = C.c_void_p()
    assert lib.granite_ccz4_create(C.byref(p), C.byref(h)) == -6
    assert lib.granite_ccz4_create(None, C.byref(h)) == -1
    assert lib.granite_ccz4_destroy(None) == 0


def test_null_context_is_an_error_everywhere(lib):
    """Every entry point that takes a context answers a null one with
    GRANITE_ERR_INVALID before touching a device (no GPU needed)."""
    import granite_b200 as gb
    d = gb.block_desc((8, 8, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    buf = (C.c_double * 8)()
    cnt = C.c_longlong()
    t = C.c_double()
    hz = gb._Horizon()
    hp = gb._HorizonParams()
    lib.granite_ccz4_default_horizon_params(C.byref(hp))
    assert (hp.max_iterations, hp.tolerance, hp.angular_resolution, hp.initial_guess_radius) == (200, 1e-10, 50, 1.0)
    lib.granite_ccz4_default_horizon_params(None)  # tolerated
    f = C.c_double  # this library handle has no argtypes: doubles go in explicitly
    calls = [
        lib.granite_ccz4_regrid_add(None, C.byref(d), 1),
        lib.granite_ccz4_tag_count(None, 0, 0, f(0.1), C.byref(cnt)),
        lib.granite_ccz4_level_time(None, 0, C.byref(t)),
        lib.granite_ccz4_hierarchy_step_regrid(None, f(0.1), 0, 0, 0, None, None),
        lib.granite_ccz4_enable_matter(None, 1),
        lib.granite_ccz4_upload_primitives(None, 0, buf),
        lib.granite_ccz4_set_primitives_device(None, 0, None),
        lib.granite_ccz4_matter_sources_host(None, C.byref(d), buf, buf, buf, buf, buf),
        lib.granite_ccz4_matter_sources_device(None, C.byref(d), None, None, None, None, None, None),
        lib.granite_ccz4_psi4_modes(None, 0, buf, 1, 4, 8, 2, buf, None),
        lib.granite_ccz4_psi4_modes_host(None, C.byref(d), buf, buf, 1, 4, 8, 2, buf, None),
        lib.granite_ccz4_find_horizon(None, 0, C.byref(hp), buf, C.byref(hz), None),
        lib.granite_ccz4_find_horizon_host(None, C.byref(d), buf, C.byref(hp), buf, C.byref(hz), None),
        lib.granite_ccz4_find_all_horizons(None, 0, C.byref(hp), C.byref(hz), 1, None),
        lib.granite_ccz4_checkpoint_write(None, b"x", 0, f(0.0)),
        lib.granite_ccz4_checkpoint_read(None, b"x", None, None),
        lib.granite_ccz4_upload_all(None, None),
        lib.granite_ccz4_download_all(None, None),
        lib.granite_ccz4_download_all_async(None, None),
    ]
    assert calls == [-1] * len(calls)
    n = C.c_int()
    assert lib.granite_ccz4_checkpoint_header(b"/nonexistent/checkpoint", None, None, None, None, 0, C.byref(n)) == -1


def test_gridblock_layout_matches_reference_conventions():
    import granite_b200 as gb
    b = gb.GridBlock(3, 1, (6, 5, 4), (-1.0, 0.0, 2.0), (2.0, 1.0, 3.0), 4, 22)
    g = Geom((6, 5, 4), (-1.0, 0.0, 2.0), (2.0, 1.0, 3.0))
    assert b.array.shape == g.shape
    assert b.totalSize() == g.cells
    for d, n in enumerate((6, 5, 4)):
        for idx in range(n + 8):
            assert b.x(d, idx) == g.x(d, idx)
    # flat index = var*stride + i + nx*(j + ny*k) (grid.hpp:109-116)
    b.set(5, 2, 3, 1, 7.0)
    stride = 14 * 13 * 12
    assert b.flatBuffer()[5 * stride + 2 + 14 * (3 + 13 * 1)] == 7.0


def test_initial_data_matches_oracle(oracle_lib):
    import granite_b200 as gb
    g = Geom((12, 10, 8), (-3.0, -2.5, -2.0), (3.0, 2.5, 2.0))
    b = gb.GridBlock(0, 0, g.n, g.lo, g.hi)
    gb.brill_lindquist(b, [0.5, 0.4], [[0.3, 0.0, 0.0], [-0.4, 0.1, 0.0]], r_floor=0.2)
    ref = oracle_lib.init_brill_lindquist(g, [0.5, 0.4], [[0.3, 0.0, 0.0], [-0.4, 0.1, 0.0]], 0.2)
    np.testing.assert_allclose(b.array, ref, rtol=1e-14, atol=1e-15)
    gw = Geom((16, 4, 4), (-0.5, -0.5, -0.5), (0.5, -0.25, -0.25))
    b = gb.GridBlock(0, 0, gw.n, gw.lo, gw.hi)
    gb.gauge_wave(b, -0.1, 1.0)
    np.testing.assert_allclose(b.array, oracle_lib.init_gauge_wave(gw, -0.1, 1.0), rtol=1e-14,
                               atol=1e-15)


def _prototypes():
    """{name: parameter count} of every granite_ccz4_* prototype in the header."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(granite_ccz4_\w+)\s*\(([^;{]*?)\)\s*;", text):
        args = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_ctypes_argtypes_match_the_header():
    """Every argtypes list the Python mirror sets has the header's arity."""
    import granite_b200 as gb
    lib = gb.load_library()
    protos = _prototypes()
    assert set(protos) == set(declared_functions())
    checked = 0
    for name, n in protos.items():
        at = getattr(lib, name).argtypes
        if at is not None:
            assert len(at) == n, (name, len(at), n)
            checked += 1
    assert checked >= 40


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """Sizes and field offsets of the ctypes mirrors equal the C compiler's."""
    import granite_b200 as gb
    mirrors = {"granite_ccz4_params": gb._Params, "granite_block_desc": gb._BlockDesc,
               "granite_horizon_params": gb._HorizonParams, "granite_horizon": gb._Horizon}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "granite_ccz4.h"', 'int main(void) {']
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["/usr/bin/gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, field, v = line.split()
        got[(cname, field)] = int(v)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_missing_library_is_an_error_not_a_fallback(monkeypatch, tmp_path):
    """Without libgranite_ccz4.so the package raises; there is no other path."""
    import granite_b200 as gb
    from granite_b200 import build
    monkeypatch.setattr(gb, "_LIB", None)
    monkeypatch.setattr(build, "LIB", str(tmp_path / "libgranite_ccz4.so"))
    with pytest.raises(gb.GraniteError):
        gb.load_library(build_if_missing=False)


def test_stage_configs_and_classes_without_a_device():
    """The TMA configuration table and the block-size classes of the autotuner
    are host data: readable without a GPU."""
    import granite_b200 as gb
    for k in range(gb.STAGE_CONFIGS):
        info = gb.stage_config_info(k)
        assert info["tile"][:2] == (16, 4) and info["tile"][2] in (2, 4)
        assert info["ring_slots"] in (2, 3, 4)
        assert info["ctas_per_sm"] in (1, 2, 3)
        assert info["items_per_barrier"] in (1, 2) and info["ring_slots"] > info["items_per_barrier"]
        if info["ctas_per_sm"] == 3:
            # the ring and the stage-input column of one CTA fit three times in
            # an SM's 228 KB of shared memory (with 7.5 KB per CTA for static
            # buffers and the per-CTA reservation)
            nt = 64 * info["tile"][2]
            dyn = info["ring_slots"] * 24 * 12 * (info["tile"][2] + 8) * 8 + 256
            dyn += 22 * nt * 8 if info["shared_input"] else 0
            assert not info["shared_hessian"] and 3 * (dyn + 7680) <= 228 * 1024, (k, info)
    assert [gb.stage_config_info(k)["ctas_per_sm"] for k in (6, 7)] == [3, 3]
    assert [gb.stage_config_info(k)["items_per_barrier"] for k in range(gb.STAGE_CONFIGS)] == \
        [1] * 8 + [2] * 3 + [1] * 4 + [2] * 3
    rem = [k for k in range(gb.STAGE_CONFIGS) if gb.stage_config_info(k)["x_remainder_tiles"]]
    assert rem == [11, 12, 13, 14, 15, 16, 17]
    assert [gb.stage_config_info(k)["tile"][2] for k in rem] == [2, 2, 2, 2, 4, 4, 2]
    with pytest.raises(gb.GraniteError):
        gb.stage_config_info(gb.STAGE_CONFIGS)
    assert [gb.block_stage_class((e, e, e)) for e in gb.STAGE_CLASS_EDGES] == list(range(6))
    assert gb.block_stage_class((16, 24, 32)) == 1  # cube root of the volume 22.9: nearest edge 24
    assert gb.block_stage_class((32, 32, 16)) == 1  # 25.4 -> 24
    assert gb.block_stage_class((200, 200, 200)) == 5
