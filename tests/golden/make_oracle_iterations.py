"""Records the CPU oracle's full-solve iteration counts for the bench workloads.

bench.py's reference arm times the oracle on a bounded sample of iterations and
extrapolates to the iteration count of a complete solve; this script runs that
complete solve (CG + SSOR with the reference's multicolour ordering, X0 = 0,
tolerance 1e-8) and writes tests/golden/oracle_iterations.json.

    python tests/golden/make_oracle_iterations.py 100,100,100
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from frontistr_b200.mesh import box_system  # noqa: E402
from oracle_ctypes import Oracle  # noqa: E402


def main(meshes, precond=1, tol=1e-8):
    path = os.path.join(HERE, "oracle_iterations.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for mesh in meshes:
        nx, ny, nz = (int(v) for v in mesh.split(","))
        m = box_system(nx, ny, nz)
        orc = Oracle(m)
        pc = orc.precond(precond, 10, 1.0, 1)
        t0 = time.time()
        res = pc.cg(m.B, maxit=20000, tol=tol)
        dt = time.time() - t0
        assert res["error"] == 0
        out["%d,%d,%d/%d" % (nx, ny, nz, precond)] = res["iter"]
        print(mesh, precond, res["iter"], res["resid"], "%.1f s" % dt, flush=True)
    json.dump(out, open(path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["100,100,100"])
