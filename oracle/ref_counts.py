"""Reference-order traversal counts of bench.py's workloads (test and bench
infrastructure, CPU only).

Walks every shadow ray of the workload through the oracle's restatement of
the reference's stackless traversal (src/GPUBVH.jl:202-285) and prints the
number of rays, box tests and triangle tests in the reference's own order --
the algorithmic work bench.py credits the traversal kernels with
(REF_COUNTS).  Usage: python oracle/ref_counts.py {medium,full} [threads]
(full: about 13 minutes on 8 cores, 15 GB of host memory)."""
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
from conftest import load_pkg  # noqa: E402

from oracle import pyoracle as orc  # noqa: E402


def main():
    size = sys.argv[1] if len(sys.argv) > 1 else "medium"
    threads = int(sys.argv[2]) if len(sys.argv) > 2 else 0
    rvf = load_pkg()
    m = {"full": 60, "medium": 24}[size]
    md = rvf.meshes.cube_enclosure(m, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12)
    t = time.time()
    _, _, _, cnt = orc.solve_plain(orc.Mesh(md, [7]), 3, threads=threads)
    print(json.dumps({"size": size, "n_rays": int(cnt[1]), "node_visits": int(cnt[2]), "prim_tests": int(cnt[3]),
                      "seconds": round(time.time() - t, 1)}))


if __name__ == "__main__":
    main()
