"""Generates simg_tie.npz: a TIP3P bulk configuration (the first replica of the
seeded 256-replica uneven batch, ensemble 0: 525 molecules, rcut 11.55 A, box
24.6 A, so the per-site minimum image is active; lattice start disordered by a
seeded 0.25 A displacement) in which several site pairs
within rcut have one component within 1e-7..3e-6 A of half the box length, on
both sides.  There the per-site image (src/force_calculator.cxx:737-741) flips
the site vector by a box length, so an FP32 evaluation that rounds across L/2
takes the other image than the FP64 oracle.  The parity test evaluates this
configuration with the FP32 engine and checks it against the oracle.

Run from the repository root:  python tests/golden/make_simg_tie.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from remd_b200 import systems as S  # noqa: E402


def site_vec(r, q, L, b, i, j, k, l):
    gr = (r[i] - r[j]) * L
    gr = np.where(gr >= 0.5 * L, gr - L, gr)
    gr = np.where(gr < -0.5 * L, gr + L, gr)
    si = S.body_to_space(q[i:i + 1], b)[0, k]
    sj = S.body_to_space(q[j:j + 1], b)[0, l]
    return gr, gr + si - sj


def main():
    e = S.config4(seed=4)[0]
    st = e.states[0]
    r, q = st.r.copy(), st.q.copy()
    # the box compressed to 24.6 A (as the barostat takes it), below
    # 2 (rcut + 2 site reach) = 26.8 A, so the per-site minimum image applies
    L = np.full(3, 24.6)
    # disorder the lattice start (seeded, 0.25 A per component) so that site
    # pairs take a continuum of separations
    rng = np.random.default_rng(2026)
    r = (r + rng.normal(0.0, 0.25, r.shape) / L) % 1.0
    b = e.spec.moltype.r
    ns, rc, n = e.spec.moltype.nsite, e.spec.rcut, e.spec.nmol
    offsets = [3e-7, -3e-7, 1e-6, -1e-6, 2e-6, -2e-6, 1e-7, -1e-7, 5e-7, -5e-7, 3e-6, -3e-6]
    used = set()
    ties = []
    for i in range(n):
        if len(ties) == len(offsets) or i in used:
            continue
        for j in range(n):
            if j == i or j in used:
                continue
            gr, _ = site_vec(r, q, L, b, i, j, 0, 0)
            if gr @ gr > (rc - 0.15) ** 2:
                continue
            hit = None
            for k in range(ns):
                for l in range(ns):
                    _, rv = site_vec(r, q, L, b, i, j, k, l)
                    for ax in range(3):
                        if abs(abs(rv[ax]) - 0.5 * L[ax]) < 0.05:
                            hit = (k, l, ax)
            if hit is None:
                continue
            k, l, ax = hit
            target_off = offsets[len(ties)]
            for _ in range(6):   # move j along ax until |rv_ax| = L/2 + offset
                _, rv = site_vec(r, q, L, b, i, j, k, l)
                want = np.sign(rv[ax]) * (0.5 * L[ax] + target_off)
                r[j, ax] -= (want - rv[ax]) / L[ax]
            r[j, ax] %= 1.0
            _, rv = site_vec(r, q, L, b, i, j, k, l)
            ties.append((i, j, k, l, ax, abs(rv[ax]) - 0.5 * L[ax]))
            used.update((i, j))
            break
    for t in ties:
        print("tie i=%d j=%d sites %d-%d axis %d |x|-L/2=%+.2e A" % t)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "simg_tie.npz")
    np.savez(out, r=r, q=q, L=L, ties=np.array([t[:5] for t in ties]),
             offsets=np.array([t[5] for t in ties]), rcut=e.spec.rcut, rswitch=e.spec.rswitch)


if __name__ == "__main__":
    main()
