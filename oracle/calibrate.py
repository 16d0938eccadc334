"""Iteration counts of full oracle solves on the benchmark workload.

The CPU baseline of bench.py times a bounded sample (assembly, AMS setup,
one FGMRES iteration) on the box where it runs and scales it by the number of
inner FCG iterations a complete oracle solve needs on the same workload.
Iteration counts do not depend on the machine, so they are measured once by
this script and committed as calibration_cfg<N>.json.

    python oracle/calibrate.py 2 [freq_index ...]
"""

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from emfem_b200 import meshgen as mg  # noqa: E402


def main():
    cfg = int(sys.argv[1]) if len(sys.argv) > 1 else 2
    fidx = [int(a) for a in sys.argv[2:]] or [0]
    prob = mg.config(cfg)
    m = O.Mesh(prob.mesh)
    rp, ci = O.sparsity(m)
    obg = O.background_model(m, prob.model)
    runs = []
    for fi in fidx:
        f = float(prob.survey.freqs[fi])
        t0 = time.time()
        Cv, Mv, bdr = O.assemble(m, prob.model, f, rp, ci)
        ta = time.time() - t0
        sr, si = O.rhs_mt(m, prob.model, f, -1, obg, bdr)
        er, ei, its, st = O.solve(m, rp, ci, Cv, Mv, sr, si, 1e-8, 100)
        runs.append(dict(freq=f, mode="XY", outer=int(its), inner=int(st[1]), true_res=float(st[0]),
                         assemble_s=ta, setup_s=float(st[2]), fgmres_s=float(st[3])))
        print(json.dumps(runs[-1]), flush=True)
    out = dict(workload=prob.name, tets=prob.mesh.n_tets, edges=prob.mesh.n_edges, runs=runs,
               inner_per_rhs=sum(r["inner"] for r in runs) / len(runs),
               threads=O.num_threads(0))
    with open(os.path.join(HERE, "calibration_cfg%d.json" % cfg), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
