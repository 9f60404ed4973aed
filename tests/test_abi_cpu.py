"""CPU checks of the boundary: the shared library loads and exports every
function include/aphid_gpu.h declares; the host-side model code agrees with
the oracle.  No GPU calls."""
import ctypes
import os
import re

import numpy as np
import pytest

from aphid_git_b200 import build, model
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(aphid_(?:gpu|unet)_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(build.build())
    names = declared_functions()
    assert len(names) >= 9
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_spacings_match_oracle():
    rng = np.random.default_rng(0)
    xn = np.cumsum(rng.uniform(1, 5, 11))
    d, dc = model.spacings(xn)
    d0, dc0 = O.spacings(xn)
    assert np.array_equal(d, d0) and np.array_equal(dc, dc0)


@pytest.mark.parametrize("mode", [1, 2, 3, 5])
def test_gen_rhs_matches_oracle(mode):
    rng = np.random.default_rng(mode)
    xn = np.concatenate([[-300.0, -200.0, -100.0], [0.0], [120.0, 250.0, 400.0]])
    yn = np.cumsum(rng.uniform(50, 90, 6)) - 200.0
    yn[2] = 0.0
    zn = np.array([-300.0, -100.0, 0.0, 50.0, 120.0, 300.0])
    dips = [("+X", 2, 3, 3), ("-X", 3, 2, 4), ("+Y", 1, 2, 2), ("-Y", 4, 6, 3), ("+Z", 5, 5, 5),
            ("-Z", 2, 2, 1), ("+W", 1, 1, 1), ("+X", 7, 1, 1), ("-Z", 3, 3, 6)]
    g = O.Grid(xn, yn, zn)
    b0, s0 = O.gen_rhs(g, mode, dips if mode == 5 else ())
    b1, s1 = model.gen_rhs(xn, yn, zn, mode, dips if mode == 5 else ())
    assert s0 == s1
    assert np.allclose(b0, b1, rtol=1e-15, atol=0)


@pytest.mark.parametrize("mode", ["R", "C", "D", "I"])
def test_sigma_hat_matches_oracle(mode):
    rng = np.random.default_rng(7)
    n = 50
    a = [rng.uniform(0.01, 1, n).astype(np.float32) for _ in range(5)]
    w = 2 * np.pi * 37.0
    s0 = O.sigma_hat(mode, w, *a)
    s1 = model.sigma_hat(mode, w, *a)
    assert np.allclose(s0, s1, rtol=1e-14, atol=0)


def test_mesh_file_roundtrip(tmp_path):
    m = model.make_model("halfspace32")
    p = tmp_path / "aphid.mesh"
    model.write_mesh(p, m.xn, m.yn, m.zn, m.sig_re)
    r = model.read_mesh(p, "R")
    assert np.allclose(r["xn"], m.xn, rtol=1e-6) and len(r["zn"]) == len(m.zn)
    assert np.array_equal(r["sig_re"], m.sig_re.ravel(order="F"))


def test_reference_example_files_parse(tmp_path):
    # layouts of serial/aphid.input and parallel/aphid_mpi.* (formats only)
    (tmp_path / "aphid.input").write_text(
        "=\nAPHID Input File\n=\n2         !! operational mode\n1.d-12    !! QMR target\n"
        "2000      !! max QMR iterates\n1.d-02    !! frequency [Hz]\nR         !! model\n")
    inp = model.read_input(tmp_path / "aphid.input")
    assert inp["oper_mode"] == 2 and inp["qmr_target"] == 1e-12 and inp["qmr_max_it"] == 2000
    assert inp["freq"] == 1e-2 and inp["csig_flag"] == "R"
    (tmp_path / "aphid_mpi.freq").write_text("=\nfreqs\n=\n2   ! n\n0.01\n0.1\n1.0\n")
    assert list(model.read_mpi_freq(tmp_path / "aphid_mpi.freq")) == [0.01, 0.1]
    (tmp_path / "aphid_mpi.source").write_text(
        "=\nAPHID: list\n=\n2 ! arrays\n\n=\ndipole array definition\n=\n1 ! n\n+X 50 50 51 ! d\n"
        "\n=\ndipole array definition\n=\n2 ! n\n+Y 50 50 51\n+Y 50 52 51\n")
    arrs = model.read_mpi_source(tmp_path / "aphid_mpi.source")
    assert arrs == [[("+X", 50, 50, 51)], [("+Y", 50, 50, 51), ("+Y", 50, 52, 51)]]
    sy = model.sweep_systems([0.1, 1.0], "CS", arrs)
    assert [s["freq"] for s in sy] == [0.1, 1.0, 0.1, 1.0] and sy[2]["dipoles"] == tuple(arrs[1])


def test_synthetic_models_shapes():
    m = model.make_model("hetero96")
    assert m.dims == (97, 97, 97) and m.sig_re.shape == (96, 96, 96)
    earth = m.sig_re[:, :, 8:]
    assert earth.min() >= 1e-4 * 0.999 and earth.max() <= 10.0 * 1.001
    assert np.all(m.sig_re[:, :, :8] == np.float32(1e-8))
    s = model.make_model("sweep128")
    assert len(s.systems()) == 96


def _c_struct_fields(header, name):
    import re
    m = re.search(r"typedef struct \{([^{}]*)\} " + name + ";", header)
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "int a, b", "const char *p", "long long n", "int r[2]": the last
        # word of each comma-separated part is a field name
        fields += [part.replace("*", " ").split()[-1].split("[")[0] for part in decl.split(",")]
    return fields


def _fortran_type_fields(src, name):
    import re
    m = re.search(r"type, bind\(C\) :: " + name + r"\n(.*?)end type " + name, src, re.S)
    fields = []
    for line in m.group(1).splitlines():
        if "::" in line:
            fields += [n.strip().split("(")[0] for n in line.split("::", 1)[1].split(",")]
    return fields


def test_fortran_binding_types_match_the_c_structs():
    """The ISO_C_BINDING module's bind(C) types carry the C structs' fields in
    the same order (a missing trailing field makes the library read or write
    past the Fortran variable)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "include", "aphid_gpu.h")) as f:
        header = f.read()
    with open(os.path.join(root, "aphid_git_b200", "fortran", "aphid_gpu_mod.f90")) as f:
        src = f.read()
    for name in ("aphid_opts", "aphid_info", "aphid_sweep_opts", "aphid_source"):
        assert _fortran_type_fields(src, name) == _c_struct_fields(header, name), name
