"""Copies the reference's ASCII pi mesh (tests/data/pi of
suvarchal/fesom2_tracer_dwarf: the files mesh_setup reads on one process) into
this directory, gzip-compressed byte for byte, as the fixture of the mesh
reader and domain decomposition tests.  Run once where the reference checkout is available:

    python tests/golden/pi/make_pi_fixture.py /path/to/fesom2_tracer_dwarf
"""
import gzip
import sys
from pathlib import Path

FILES = ["nod2d.out", "elem2d.out", "aux3d.out", "edgenum.out", "edges.out", "edge_tri.out", "elvls.out",
         "nlvls.out"]
# the partition directories for 2 and 8 parts (rpart.out, the my_list and
# com_info files; stored as dist_2__rpart.out.gz, ..., "__" standing for "/")
PARTITIONS = [f"dist_{n}/{f}" for n in (2, 8)
              for f in ["rpart.out"] + [f"{kind}{r:05d}.out" for kind in ("my_list", "com_info") for r in range(n)]]


def main(reference_root: str) -> None:
    src = Path(reference_root) / "tests" / "data" / "pi"
    dst = Path(__file__).resolve().parent
    for name in FILES + PARTITIONS:
        data = (src / name).read_bytes()
        out = dst / (name.replace("/", "__") + ".gz")
        with gzip.GzipFile(out, "wb", mtime=0) as f:
            f.write(data)
        print(f"{name}: {len(data)} bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
