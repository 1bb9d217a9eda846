"""Runs one workload through the compiled reference and writes its results (test helper of
tests/test_gpu_adapter.py).  With AUSAXS_REF_LIB=libausaxs_ref_gpu.so the same reference code runs
with its Simple, partial and symmetry managers over the device calculator and with the device FFAvg
manager; without it, on the reference's own CPU classes.  Each library runs in a process of its own.

usage: python tests/adapter_run.py <out.npz>"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import py as O  # noqa: E402

Q_AXIS = (1e-4, 0.5)


def molecule(seed, sizes, waters=0):
    rng = np.random.default_rng(seed)
    xyz = np.concatenate([rng.normal(0, 6, (n, 3)) + rng.uniform(-15, 15, 3) for n in sizes])
    ff = rng.choice([3, 7, 11, 12], len(xyz), p=[0.63, 0.17, 0.19, 0.01]).astype(np.int32)
    charge = {3: 5.997198, 7: 6.996361, 11: 7.999706, 12: 15.989624}
    w = np.array([charge[int(t)] for t in ff]) * rng.uniform(0.8, 1.2, len(xyz))
    wat = rng.normal(0, 12, (waters, 3))
    return O.RefMolecule(xyz, w, ff, wat, np.full(waters, 8.999659), body_sizes=sizes, volume=40.0 * len(xyz))


def main(out):
    O.ref(4)
    O.ref_set_axes(0.25, 8000, Q_AXIS[0], Q_AXIS[1])
    O.ref_set_simple_exv(False)
    res = {"adapter": np.int32(O.ref().ref_adapter_build())}
    # SymmetryManagerMT: one body with a cyclic and one with a polyhedral symmetry, waters
    for name, sym, tr in (("c3", "c3", 9.0), ("tetra", "tetrahedral", 11.0)):
        m = molecule(3 if name == "c3" else 4, [260, 140], waters=60)
        m.add_symmetry(0, sym, tr, 0.4)
        m.set_manager("symmetry")
        h = m.calculate()
        res[f"sym_{name}_tot"], res[f"sym_{name}_d"] = h.total()
        q, I, _, _ = h.debye()
        res[f"sym_{name}_I"] = I
    # HistogramManagerMT (Simple) and PartialHistogramManagerMT through two rigid moves
    m = molecule(5, [300, 200, 150], waters=80)
    m.set_manager("mt")
    h = m.calculate()
    res["mt_aa"], res["mt_aw"], res["mt_ww"] = h.simple()
    res["mt_tot"], res["mt_d"] = h.total()
    res["mt_I"] = h.debye()[1]
    m = molecule(6, [300, 200, 150], waters=80)
    m.set_manager("partial")
    rng = np.random.default_rng(7)
    for step in range(3):
        if step:
            th = rng.uniform(0, 0.3)
            R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
            m.move_body(int(rng.integers(0, 3)), R, rng.uniform(-2, 2, 3))
        h = m.calculate()
        res[f"partial{step}_tot"], res[f"partial{step}_d"] = h.total()
    # FFAvg: the device manager in the adapter build, the reference's own on the CPU
    m = molecule(8, [700], waters=150)
    m.set_manager("gpu_ffavg" if res["adapter"] else "ffavg")
    h = m.calculate()
    res["ff_aa"], res["ff_aw"], res["ff_ww"] = h.ff()
    res["ff_tot"], res["ff_d"] = h.total()
    q, I, prof, _ = h.debye()
    res["ff_q"], res["ff_I"], res["ff_prof"] = q, I, prof
    np.savez(out, **res)


if __name__ == "__main__":
    main(sys.argv[1])
