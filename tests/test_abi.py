"""C ABI of the product library: every entry point declared in include/*.h is
exported, host-only entry points behave, argument errors are reported as status
codes (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from falm_b200 import _lib, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char \*|long long)\s*(falm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib_built):
    lib = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_abi_version(lib_built):
    assert _lib.load().falm_abi_version() == 1


def test_null_arguments_are_rejected(lib_built):
    lib = _lib.load()
    assert lib.falm_create(None, 0, None) == 1
    assert lib.falm_destroy(None) == 1
    assert lib.falm_cfd_init(None, 1e3, 1, 1, 0.1) == 1
    assert lib.falm_step(None, None, 0.1, 0.0, None, None) == 1
    assert lib.falm_eq_solve(None, None, None, None, None, None, None) == 1
    assert lib.falm_alm_build_aps(0, None, None, None, None, None, 0, 0, 0, 1.0, 0.0, None, None, None, None, None) == 1


def test_build_aps_host_entry_point(lib_built):
    from falm_b200.api import build_aps
    st = cases.blade_stations()
    got = build_aps(st, 1, 3, 32, 1.0, 0.0)
    ref = cases.build_aps_py(st, 96, 32, 1.0, 0.0)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k])


def test_inflow_box_statistics():
    box = cases.inflow_box(24, 20, 0.05, nb=16, corr=8, seed=cases.INFLOW_SEED)
    assert box.shape == (3, 16, 20, 24)
    np.testing.assert_allclose(box.reshape(3, -1).std(axis=1), 0.05, rtol=1e-12)
    again = cases.inflow_box(24, 20, 0.05, nb=16, corr=8, seed=cases.INFLOW_SEED)
    np.testing.assert_array_equal(box, again)


def test_index_file_host_entry_point(lib_built, tmp_path):
    """falm_io_write_index_file renders FalmIO::writeIndexFile's object as
    nlohmann::json's dump(2) does: sorted keys, two-space indent, no final
    newline, and each double as its shortest round-trip digits laid out by the
    library's rules (fixed point for decimal exponents -4 < n <= 15, ".0" on
    integral values, else d.ddde+XX)."""
    import json
    from falm_b200 import api
    snaps = [(100, 1.5, False), (200, 3.0, True), (300, 0.1 + 0.2, True), (7, 1e-05, False), (8, 0.0001, False)]
    api.write_index_file(tmp_path / "a.json", (64, 32, 16), 2, snaps, dsize=4)
    text = (tmp_path / "a.json").read_text()
    obj = {"dataType": "float32", "global": [64, 32, 16], "guidePoint": 2,
           "outputSteps": [dict({"step": s, "time": t}, **({"timeAvg": 1} if a else {})) for s, t, a in snaps],
           "ranks": [{"offset": [0, 0, 0], "rank": 0, "voxel": [64, 32, 16]}], "variables": ["u", "v", "w", "p"]}
    assert text == json.dumps(obj, indent=2, sort_keys=True)
    # the cases where Python's float repr and the library's layout differ, by the rules above
    cases_ = {1e15: "1e+15", 2.5e15: "2.5e+15", 123456789012345.6: "123456789012345.6", 1e16: "1e+16",
              5e-324: "5e-324", 1.7976931348623157e308: "1.7976931348623157e+308", -2.0: "-2.0", 0.0: "0.0",
              100.0: "100.0", 1e-4: "0.0001", 1.25e-5: "1.25e-05", 1e100: "1e+100"}
    api.write_index_file(tmp_path / "b.json", (4, 4, 4), 2, [(q, v, False) for q, v in enumerate(cases_)])
    got = [line.split(": ")[1] for line in (tmp_path / "b.json").read_text().splitlines() if '"time"' in line]
    assert got == list(cases_.values())
    # an empty snapshot list has no outputSteps key, as the reference's object
    api.write_index_file(tmp_path / "c.json", (4, 4, 4), 2, [])
    assert "outputSteps" not in json.loads((tmp_path / "c.json").read_text())
    lib = _lib.load()
    assert lib.falm_io_write_index_file(b"/nonexistent/dir/x.json", 4, 4, 4, 2, None, None, None, 0, 8) == 1
    assert lib.falm_io_write_index_file(str(tmp_path / "d.json").encode(), 4, 4, 4, 2, None, None, None, 0, 2) == 1


def test_control_volume_reader_host_entry_point(lib_built, tmp_path):
    """falm_io_read_cv_file reads FalmIO::writeControlVolumeFile's text layout."""
    from falm_b200 import api
    g = cases.stretched_grid(10, 6, 5, 0.1)
    with open(tmp_path / "g.cv", "w") as f:
        f.write(f"{g.sx} {g.sy} {g.sz} {g.gc}\n")
        for c, h in ((g.x, g.hx), (g.y, g.hy), (g.z, g.hz)):
            for a, b in zip(c, h):
                f.write("\t%.15e\t%.15e\n" % (a, b))
    dims, x, hx, y, hy, z, hz = api.read_cv_file(tmp_path / "g.cv")
    assert dims == (g.sx, g.sy, g.sz, g.gc)
    for a, b in ((x, g.x), (hx, g.hx), (y, g.y), (hy, g.hy), (z, g.z), (hz, g.hz)):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=0)
    (tmp_path / "bad.cv").write_text("4 4\n")
    with pytest.raises(_lib.FalmError):
        api.read_cv_file(tmp_path / "bad.cv")


REF_SO = os.path.join(ROOT, "oracle", "_ref", "libfalmref.so")


def _node_files(d, xs, ys, zs):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "mesh.json"), "w") as f:
        f.write('{\n    "coordinatePoint":"node"\n}')
    for name, v in (("x.txt", xs), ("y.txt", ys), ("z.txt", zs)):
        with open(os.path.join(d, name), "w") as f:
            f.write(f"{len(v)}\n" + "".join("%.15e\n" % a for a in v))


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("mode", ["cell", "innerNode"])
def test_mesher_matches_reference(lib_built, tmp_path, mode):
    """falm_mesh_build against the reference's own Mesher::build_mesh (compiled
    into oracle/_ref, host code only): byte-identical control-volume files for
    stretched node coordinates, with a 2-node axis for the constant-width branch
    of "cell"; the file reads back through falm_io_read_cv_file."""
    from falm_b200 import api
    xs = np.cumsum(np.concatenate([[-1.0], 0.05 * 1.07 ** np.arange(30)]))
    ys = np.linspace(-0.5, 0.7, 13)
    zs = np.array([0.0, 0.25]) if mode == "cell" else np.cumsum(np.concatenate([[0.0], 0.02 * 1.1 ** np.arange(9)]))
    src = str(tmp_path / "mesh")
    _node_files(src, xs, ys, zs)
    ref = ctypes.CDLL(REF_SO)
    ref.ref_build_mesh.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    for gc in (2, 3):
        a, b = str(tmp_path / f"ref{gc}.cv"), str(tmp_path / f"b200{gc}.cv")
        assert ref.ref_build_mesh(mode.encode(), src.encode(), a.encode(), gc) == 0
        api.build_mesh(mode, src, b, gc)
        assert open(a, "rb").read() == open(b, "rb").read()
        dims, x, hx, y, hy, z, hz = api.read_cv_file(b)
        assert dims[3] == gc
        if mode == "cell":
            assert dims[:3] == (len(xs) - 1 + 2 * gc, len(ys) - 1 + 2 * gc, len(zs) - 1 + 2 * gc)
            np.testing.assert_allclose(hx[gc:-gc], np.diff(xs), rtol=1e-14)
        else:
            assert dims[:3] == (len(xs) + 2 * (gc - 1), len(ys) + 2 * (gc - 1), len(zs) + 2 * (gc - 1))
            np.testing.assert_allclose(x[gc - 1:len(x) - gc + 1], xs, rtol=0, atol=1e-15)
    with pytest.raises(_lib.FalmError):
        api.build_mesh("face", src, str(tmp_path / "x.cv"), 2)


def test_class_shim_compiles(tmp_path):
    """Every class of the C++ shim (include/falm_b200.hpp) instantiated in both
    precisions, including the slab (Context::slab, CPMComm) and RMCP
    (Rmcp::RmcpAlm) surfaces: a syntax-only compile against the CUDA headers."""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc")
    if nvcc is None:
        pytest.skip("no CUDA toolkit")
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
    src = tmp_path / "shim.cpp"
    src.write_text(r'''
#include "falm_b200.hpp"
using namespace Falm;
template <typename Real> void use(Context &ctx, const falm_transport &t, const falm_rmcp_desc &rd) {
    ctx.slab(0, 2, 0, 64, t);
    FalmCFD<Real> cfd(ctx);
    FalmEq<Real> eq(ctx);
    Alm::AlmHandler<Real> alm(ctx);
    Rmcp::RmcpAlm<Real> rmcp(ctx);
    CPMComm<Real> comm(ctx);
    Int3 dom{{8, 8, 8}};
    Matrix<Real> u(dom, 3), ff(dom, 3), p(dom, 1);
    Matrix<int> flag(dom, 1);
    rmcp.init(rd);
    rmcp.SetALMFlag(flag, u, ff, Real(0));
    rmcp.ALM(u, ff, Real(0));
    comm.IExchange6Face(p.dev.ptr, 1, 2, 0);
    comm.Wait6Face();
    comm.PostExchange6Face();
    (void)FalmMV<Real>::DotProduct(ctx, p, p);
    (void)ctx.cpm.validNeighbour(CPM::ZPLUS);
    (void)cfd; (void)eq; (void)alm;
}
template void use<double>(Context &, const falm_transport &, const falm_rmcp_desc &);
template void use<float>(Context &, const falm_transport &, const falm_rmcp_desc &);
''')
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                        str(src)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
