"""Generate the committed fixtures in tests/golden from the CPU oracle.

Run:  python tests/golden/make_golden.py
The reference ships no golden vectors and cannot be compiled here, so these fixtures pin
the oracle's own outputs (regression anchors), not the reference's; the inputs are the
seeded synthetic tangles of nuvort_b200.rings.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from helpers import config0_params, config1_params, tangle  # noqa: E402


def config0_bs():
    return tangle(0, 0.002, n_rings=8), config0_params(), "velocity"


def config1_tree_small():
    return tangle(1, 0.001, n_points=2048), config1_params("Tree"), "velocity"


CASES = {"config0_bs": config0_bs, "config1_tree_small": config1_tree_small}


def main():
    from oracle import Oracle
    for name, fn in CASES.items():
        st, p, kind = fn()
        o = Oracle(p, st)
        out = {"u": o.calc_velocity()}
        if name == "config0_bs":
            o2 = Oracle(p, st)
            o2.step(40)
            d = o2.download()
            out.update(nsteps=np.int32(40), x_after=d.x, infront_after=d.infront,
                       events=np.array(o2.events(), dtype=np.int32).reshape(-1, 4))
        else:
            o.stage("ghostp")
            o.stage("construct_tree")
            tr = o.tree_dump()
            out.update(tree_cent=tr["cent"], tree_pcount=tr["pcount"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: getattr(v, "shape", v) for k, v in out.items()})


if __name__ == "__main__":
    main()
