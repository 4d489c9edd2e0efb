"""Regenerates tests/golden/ref_meshes.npz from libsupermesh's own test data.

Reads the Triangle/TetGen meshes of firedrakeproject/libsupermesh
src/tests/data (the small files and the 2D_0_01 / 3D_0_05 archives that the
reference's CMake extracts at configure time, CMakeLists.txt:313-319) and
stores them as float64 positions + 0-based int32 element lists, so the
parity tests can run where the reference checkout is absent.

Usage: python tests/golden/make_fixtures.py /path/to/libsupermesh
"""
import sys
import tarfile
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from libsupermesh_b200.meshes import read_mesh  # noqa: E402

SMALL = ["triangle.1", "triangle.2", "tet", "square.1", "square.2", "square.3", "square.4", "cube.1",
         "cube.2", "cube.3", "cube.4", "line.1", "line.2"]
ARCHIVES = {"2D_0_01.tar.bz2": ["triangle_0_01", "square_0_01"],
            "3D_0_05.tar.bz2": ["pyramid_0_05", "cube_0_05"]}


def main(ref: Path) -> None:
    data = ref / "src" / "tests" / "data"
    out = {}
    for name in SMALL:
        pos, en = read_mesh(data / name)
        out[f"{name}/positions"] = pos
        out[f"{name}/enlist"] = en
    with tempfile.TemporaryDirectory() as tmp:
        for arc, names in ARCHIVES.items():
            with tarfile.open(data / arc) as tf:
                for n in names:
                    for ext in (".node", ".ele"):
                        tf.extract(n + ext, tmp)
            for n in names:
                pos, en = read_mesh(Path(tmp) / n)
                out[f"{n}/positions"] = pos
                out[f"{n}/enlist"] = en
    np.savez_compressed(Path(__file__).with_name("ref_meshes.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_fixtures.py /path/to/libsupermesh")
    main(Path(sys.argv[1]))
