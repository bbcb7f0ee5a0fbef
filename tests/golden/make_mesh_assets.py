"""Copy the reference's two mesh test assets (test/assets/square.obj and square.stl, 73 and 379
bytes) into tests/golden/ so the import checks of test/MeshInterop.jl:16-22 run without the
reference tree.  Run once where the reference is mounted:

    python tests/golden/make_mesh_assets.py /path/to/CombinatorialSpaces.jl
"""
import pathlib
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    src = pathlib.Path(ref_root) / "test" / "assets"
    for name in ("square.obj", "square.stl"):
        shutil.copyfile(src / name, HERE / name)
        print("wrote", HERE / name)


if __name__ == "__main__":
    main(sys.argv[1])
