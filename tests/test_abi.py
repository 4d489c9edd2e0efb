"""The CUDA library loads and exports every function include/*.h declares
(CPU-only: no device calls)."""
import ctypes
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(libsupermesh_\w+)\s*\(", re.M)


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in DECL.finditer(text):
            line = text[m.start():text.index("(", m.start())]
            if "static" in line or "#define" in line:
                continue
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    sys.path.insert(0, str(ROOT))
    from libsupermesh_b200 import build

    build.build()
    return ctypes.CDLL(str(build.OUT))


def test_headers_declare_the_reference_api():
    names = declared_symbols()
    # the 14 entries of libsupermesh-c.h upstream
    ref = {"libsupermesh_sort_intersection_finder_set_input", "libsupermesh_sort_intersection_finder_query_output",
           "libsupermesh_sort_intersection_finder_get_output", "libsupermesh_tree_intersection_finder_set_input",
           "libsupermesh_tree_intersection_finder_query_output", "libsupermesh_tree_intersection_finder_get_output",
           "libsupermesh_intersect_tris_real", "libsupermesh_intersect_tets_real", "libsupermesh_triangle_area",
           "libsupermesh_tetrahedron_volume", "libsupermesh_interval_size", "libsupermesh_intersect_intervals",
           "libsupermesh_intersect_tet_hex", "libsupermesh_intersect_tri_quad"}
    assert ref <= names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_cuda(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "libsupermesh_b200" / "lib" / "libsupermesh.so")],
                         capture_output=True, text=True, check=True).stdout
    assert "libsupermesh_gpu_supermesh" in out


def test_context_create_without_gpu_fails_cleanly(lib):
    """On a machine without a usable GPU the GPU API returns a status code;
    it neither crashes nor silently computes on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; covered by the gpu tests")
    h = ctypes.c_void_p()
    lib.libsupermesh_gpu_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    st = lib.libsupermesh_gpu_context_create(0, ctypes.byref(h))
    assert st == 5 and not h.value  # LSM_ERROR_CUDA


def test_legacy_api_without_gpu_aborts_loudly():
    """The drop-in entries have no status channel: like libsupermesh_abort
    they print and exit(1) when no device is usable."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import libsupermesh_b200 as L\n"
        "print(L.triangle_area([[0,0],[1,0],[0,1]]))\n" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "libsupermesh (B200) error" in r.stderr


def test_missing_library_raises_instead_of_falling_back(tmp_path):
    """Without the CUDA library every entry of the Python package raises;
    nothing computes on the CPU in its place."""
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from pathlib import Path\n"
        "import libsupermesh_b200 as L\n"
        "L._LIB = Path(%r)\n"
        "for f in (L.load, lambda: L.Context(0), lambda: L.triangle_area([[0,0],[1,0],[0,1]])):\n"
        "    try:\n"
        "        f()\n"
        "    except RuntimeError as e:\n"
        "        assert 'no CPU implementation' in str(e), e\n"
        "    else:\n"
        "        raise SystemExit('no error')\n"
        "print('ok')\n" % (str(ROOT), str(tmp_path / "missing.so")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr


def test_tuning_options_host_side(lib):
    """Options are process-wide host settings: valid values round-trip,
    invalid names/values are rejected (no GPU needed)."""
    import libsupermesh_b200 as L

    for name, vals in {"tri_blocks_per_sm": (16, 8), "query_block": (256, 128), "tet_screen": (0, 1),
                       "time_kernels": (1, 0), "spill_chunks": (0, 5, -1), "tet_schedule": (1, 2, 0),
                       "sched_window": (256, 8192, 1024), "fail_alloc_after": (5, -1),
                       "sort_spin_limit": (1000, 1 << 22), "sort_stall_block": (2, -1),
                       "leaf_bucket": (1, 2, 8, 4), "batch_graph": (1, 0)}.items():
        for v in vals:
            L.set_option(name, v)
            assert L.get_option(name) == v
    for bad in (("tet_clipper", 0), ("query_block", 100), ("tet_screen", 2), ("spill_chunks", -2),
                ("tet_schedule", 3), ("sched_window", 300), ("sched_window", 16384), ("sort_stall_block", 0),
                ("sort_spin_limit", 0), ("fail_alloc_after", -2), ("leaf_bucket", 3), ("batch_graph", 2),
                ("nonsense", 1)):
        with pytest.raises(L.LsmError):
            L.set_option(*bad)
