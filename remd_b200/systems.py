"""Seeded synthetic REMD systems for the benchmark configurations.

No dataset ships with the reference (its only input is test/input/gpu0000.chk),
so every workload here is generated from a seed:

  * molecules on a lattice whose O-O spacing is >= 2.9 A (bulk: simple cubic,
    3.1 A, about 1.0 g/cm^3; tube: square cross-section grid inside the
    accessible radius R-2.6 A, layers 3.0 A apart; slit: layers 2.9 A apart
    inside |z| <= w/2-1.8 A, square 3.1 A grid in x,y);
  * orientations: of 64 uniform rotations (Shoemake) per molecule, the one with
    the lowest Coulomb energy against already placed neighbours whose sites
    stay >= 1.7 A away;
  * Maxwell-Boltzmann velocities and angular velocities, then the reference's
    VelocityScaling / KillMomentum / AngVelocityScaling (src/molecules.cxx:168-307)
    so every replica starts exactly at its condition's temperature.

Periodic lengths follow from the lattice (about 1.0 g/cm^3), not from the
nominal lengths of configurations 1 and 2, which would pack water at about
2.2x and 2.45x liquid density; any periodic length below 2*rcut+2 A is raised
to that value so the minimum-image convention holds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .inputs import (ELE, UNIT_COULOMB, UNIT_PRESS, UNIT_TEMP, ReplicaState, SystemSpec,
                     load_model, moltype_path)

WALL_SGM, WALL_EPS, WALL_RHO = 3.277, 0.3886, 0.38016
BULK_MODULUS = 2.2e9 / UNIT_PRESS   # liquid water, reduced; only sizes the barostat mass


@dataclass
class Ensemble:
    """One REMD system: a T x P grid of replicas of the same molecules."""
    name: str
    spec: SystemSpec
    ntemp: int
    npress: int
    T: np.ndarray                 # reduced, per replica (REMDInfo::temperature)
    P: np.ndarray                 # reduced, per replica
    states: list = field(default_factory=list)

    @property
    def nreplica(self):
        return self.ntemp * self.npress


def conditions_geometrical(ntemp, npress, tmin_K, tmax_K, pmin_Pa, pmax_Pa):
    """REMDInfo::SetConditionGeometrical (src/remdinfo.cxx:348-359), including its
    single-precision powf ladder."""
    tmax, tmin = tmax_K / UNIT_TEMP, tmin_K / UNIT_TEMP
    pmax, pmin = pmax_Pa / UNIT_PRESS, pmin_Pa / UNIT_PRESS
    f32 = np.float32
    t = 1.0 if ntemp == 1 else float(np.power(f32(tmax / tmin), f32(1.0 / (ntemp - 1))))
    p = 0.0 if npress == 1 else (pmax - pmin) / (npress - 1)
    T = np.zeros(ntemp * npress)
    P = np.zeros(ntemp * npress)
    for j in range(npress):
        for i in range(ntemp):
            T[i + j * ntemp] = tmin * float(np.power(f32(t), f32(i)))
            P[i + j * ntemp] = pmin + p * j
    return T, P


# ------------------------------------------------------------------ geometry
def lattice(confined, nmol, wall, rc, rng):
    """Lattice start: absolute positions (A) inside the box and the box lengths."""
    minlen = 2.0 * rc + 2.0
    if confined == 0:
        n = int(math.ceil(nmol ** (1.0 / 3.0) - 1e-9))
        a = max(3.1, minlen / n)
        g = np.array([(i, j, k) for k in range(n) for j in range(n) for i in range(n)], float)
        pick = np.sort(rng.choice(len(g), nmol, replace=False))
        L = np.full(3, n * a)
        pos = (g[pick] + 0.5) * a
        return pos, L
    if confined == 1:
        racc = max(wall - 2.6, 0.0)
        a = 2.9
        m = int(racc // a)
        disc = [(i * a, j * a) for i in range(-m, m + 1) for j in range(-m, m + 1)
                if (i * a) ** 2 + (j * a) ** 2 <= racc ** 2 + 1e-9]
        k = len(disc)
        nl = int(math.ceil(nmol / k))
        c = max(3.0, minlen / nl)
        Lz = nl * c
        Lxy = 2.0 * wall + 2.0 * rc + 4.0
        pts = [(x, y, (l + 0.5) * c) for l in range(nl) for (x, y) in disc]
        pick = np.sort(rng.choice(len(pts), nmol, replace=False))
        pos = np.array(pts)[pick] + np.array([Lxy / 2, Lxy / 2, 0.0])
        return pos, np.array([Lxy, Lxy, Lz])
    # slit of width `wall` normal to z
    zacc = max(wall / 2.0 - 1.8, 0.0)
    nz = int(2 * zacc // 2.9) + 1
    zs = [(-zacc + i * 2.9) if nz > 1 else 0.0 for i in range(nz)]
    if nz > 1:
        zs = list(np.array(zs) - (zs[-1] + zs[0]) / 2.0)
    kx = int(math.ceil(math.sqrt(nmol / nz)))
    a = max(3.1, minlen / kx)
    Lxy = kx * a
    Lz = wall + 2.0 * rc + 2.0
    pts = [((i + 0.5) * a, (j + 0.5) * a, Lz / 2 + z) for z in zs for j in range(kx)
           for i in range(kx)]
    pick = np.sort(rng.choice(len(pts), nmol, replace=False))
    return np.array(pts)[pick], np.array([Lxy, Lxy, Lz])


def random_quaternions(n, rng):
    """Uniform rotations (Shoemake 1992)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    return np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                     b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)


def body_to_space(q, b):
    """Rotation of body vectors b (k,3) by unit quaternions q (n,4) -> (n,k,3),
    the map of src/rotation.h:168-187."""
    a0, a1, a2, a3 = q[:, 0:1], q[:, 1:2], q[:, 2:3], q[:, 3:4]
    x, y, z = b[None, :, 0], b[None, :, 1], b[None, :, 2]
    sx = (a0*a0 + a1*a1 - a2*a2 - a3*a3) * x + 2*(a1*a2 - a0*a3) * y + 2*(a1*a3 + a0*a2) * z
    sy = 2*(a1*a2 + a0*a3) * x + (a0*a0 - a1*a1 + a2*a2 - a3*a3) * y + 2*(a2*a3 - a0*a1) * z
    sz = 2*(a1*a3 - a0*a2) * x + 2*(a2*a3 + a0*a1) * y + (a0*a0 - a1*a1 - a2*a2 + a3*a3) * z
    return np.stack([sx, sy, sz], axis=-1)


def orientations(pos, L, body, charge, rng, min_dist=1.7, tries=64):
    """Greedy placement: for each molecule, of `tries` uniform rotations keep the
    one with the lowest Coulomb energy against the already placed neighbours
    (COM within 7 A) among those whose sites stay >= min_dist from every
    neighbour site.  This starts the lattice close to a hydrogen-bonded
    arrangement, so little heat is released in the first steps."""
    n = len(pos)
    q = np.zeros((n, 4))
    sites = np.zeros((n, len(body), 3))
    qred = charge * (ELE / UNIT_COULOMB)
    for i in range(n):
        d = pos[:i] - pos[i]
        d -= L * np.round(d / L)
        near = np.nonzero(np.einsum("ij,ij->i", d, d) < 49.0)[0]
        cand = random_quaternions(tries, rng)
        if len(near) == 0:
            q[i] = cand[0]
        else:
            sc = pos[i] + body_to_space(cand, body)                     # (t,k,3)
            ns = sites[near].reshape(-1, 3)                              # (m,3)
            nq = np.tile(qred, len(near))
            dd = sc[:, :, None, :] - ns[None, None, :, :]
            dd -= L * np.round(dd / L)
            r = np.sqrt(np.einsum("...k,...k->...", dd, dd))             # (t,k,m)
            e = np.sum(qred[None, :, None] * nq[None, None, :] / np.maximum(r, 0.5), axis=(1, 2))
            ok = r.reshape(tries, -1).min(axis=1) >= min_dist
            if ok.any():
                e = np.where(ok, e, np.inf)
            else:
                e = -r.reshape(tries, -1).min(axis=1)
            q[i] = cand[int(np.argmin(e))]
        sites[i] = pos[i] + body_to_space(q[i:i + 1], body)[0]
    return q


# ------------------------------------------------------------------ thermal state
def _Pk(q):
    """Columns P1, P2, P3 of S(q) (src/integrator.h:103-160) for q (n,4)."""
    q0, q1, q2, q3 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    P1 = np.stack([-q1, q0, q3, -q2], 1)
    P2 = np.stack([-q2, -q3, q0, q1], 1)
    P3 = np.stack([-q3, q2, -q1, q0], 1)
    return P1, P2, P3


def _kill_momentum(st: ReplicaState, confined):
    """Molecules::KillMomentum + KillAngularMomentumInTube (src/molecules.cxx:168-210)."""
    m = st.m
    mom = (st.v * m[:, None]).sum(0) / m.sum()
    if confined == 1:
        st.v[:, 2] -= mom[2]
        r = (st.r - 0.5) * st.L
        v = st.v / (st.L * st.s)
        lz = np.sum(m * (r[:, 0] * v[:, 1] - r[:, 1] * v[:, 0])) / m.sum()
        r02 = r[:, 0] ** 2 + r[:, 1] ** 2
        sel = r02 > 1.0
        st.v[sel, 0] += lz * r[sel, 1] / r02[sel] * st.L[0] * st.s
        st.v[sel, 1] -= lz * r[sel, 0] / r02[sel] * st.L[1] * st.s
    elif confined == 2:
        st.v[:, 0] -= mom[0]
        st.v[:, 1] -= mom[1]
    else:
        st.v -= mom


def thermalize(st: ReplicaState, confined, rng):
    """Maxwell-Boltzmann start scaled like VelocityScaling/AngVelocityScaling."""
    n = st.nmol
    T = st.T
    vr = rng.normal(size=(n, 3)) * np.sqrt(T / st.m)[:, None]
    st.v = vr * st.L * st.s
    _kill_momentum(st, confined)
    tra = 0.5 * np.sum(st.m[:, None] * (st.v / (st.L * st.s)) ** 2)
    st.v *= math.sqrt(1.5 * n * T / tra)
    _kill_momentum(st, confined)
    # angular: omega_k ~ N(0, T/I_k), p = 2 S(q) (0, I omega)
    om = rng.normal(size=(n, 3)) * np.sqrt(T / st.I)
    P1, P2, P3 = _Pk(st.q)
    Iw = st.I * om
    st.p = 2.0 * (P1 * Iw[:, 0:1] + P2 * Iw[:, 1:2] + P3 * Iw[:, 2:3])
    xi = np.stack([np.sum(st.p * P1, 1), np.sum(st.p * P2, 1), np.sum(st.p * P3, 1)], 1)
    xi = xi * (0.25 / st.s) / st.I
    rot = np.sum(st.I * xi * xi * 2.0)
    st.p *= math.sqrt(1.5 * n * T / rot)
    st.s, st.Ps = 1.0, 0.0
    st.Pv = np.zeros(3)


def barostat_mass(pconstant, L, wall, confined):
    """A barostat mass giving a ~0.5 ps box oscillation (omega^2 ~ 25 reduced)."""
    K, w2 = BULK_MODULUS, 25.0
    if pconstant == 1:
        return K / (L[0] * L[1] * L[2] * w2)
    if pconstant == 2:
        area = math.pi * (wall - 1.7) ** 2
        return K * area / (L[2] * w2)
    if pconstant == 3:
        return K * L[1] * (wall if confined == 2 else L[2]) / (L[0] * w2)
    return 1.0


def make_ensemble(name, model, confined, nmol, wall, rc, rs, ntemp, npress, tmin, tmax,
                  pmin, pmax, seed, nfwall=1000, tconstant=1, pconstant=None, dt=2.0,
                  tstat_mass=None, interval=100) -> Ensemble:
    rng = np.random.default_rng(seed)
    mt = load_model(model)
    if pconstant is None:
        pconstant = {0: 1, 1: 2, 2: 3}[confined]
    pos, L = lattice(confined, nmol, wall, rc, rng)
    body = mt.r
    q0 = orientations(pos, L, body, mt.charge, rng)
    m, I = mt.reduced_mass(), mt.reduced_inertia()
    Q = tstat_mass if tstat_mass is not None else max(nmol / 128.0, 0.25)
    W = barostat_mass(pconstant, L, wall, confined)
    spec = SystemSpec(nmol=nmol, moltype=mt, tconstant=tconstant, pconstant=pconstant,
                      confined=confined, dt=dt, rcut=rc, rswitch=rs,
                      nfwall=nfwall if confined else 0, wall_length=wall if confined else 0.0,
                      sgm_wall=WALL_SGM, eps_wall=WALL_EPS, rho_wall=WALL_RHO,
                      tstat_mass=Q, bstat_mass=W, interval=interval,
                      moltype_file=moltype_path(model))
    T, P = conditions_geometrical(ntemp, npress, tmin, tmax, pmin, pmax)
    ens = Ensemble(name, spec, ntemp, npress, T, P)
    for rep in range(ntemp * npress):
        rrng = np.random.default_rng([seed, rep])
        q = q0.copy()
        st = ReplicaState(r=pos / L, v=np.zeros((nmol, 3)), q=q, p=np.zeros((nmol, 4)),
                          m=np.full(nmol, m), I=np.tile(I, (nmol, 1)), Q=Q, W=W,
                          L=L.copy(), T=T[rep], P=P[rep])
        thermalize(st, confined, rrng)
        ens.states.append(st)
    return ens


# ------------------------------------------------------------------ benchmark configurations
def config1(seed=1):
    """TIP4P, N=128, tube R=6 A, rc 8.5 / rs 7.5, 4 T (240-360 K geometric) x
    4 P (0.1-200 MPa), NP thermostat Q=1 + 1-D z barostat, dt 2 fs, interval 100."""
    return [make_ensemble("config1", "tip4p", 1, 128, 6.0, 8.5, 7.5, 4, 4, 240, 360, 0.1e6,
                          200e6, seed, tstat_mass=1.0, interval=100)]


def config2(seed=2):
    """TIP4P, N=512, slit 10 A, rc 10 / rs 9, 16 T (220-380 K) x 4 P (0.1-300 MPa),
    2-D xy barostat, interval 200."""
    return [make_ensemble("config2", "tip4p", 2, 512, 10.0, 10.0, 9.0, 16, 4, 220, 380, 0.1e6,
                          300e6, seed, interval=200)]


def config3(seed=3):
    """TIP5P, N=1728, bulk simple-cubic 12^3 (37.3 A), rc 12 / rs 10, 32 T (250-450 K)
    x 4 P (0.1-400 MPa), 3-D barostat."""
    return [make_ensemble("config3", "tip5p", 0, 1728, 0.0, 12.0, 10.0, 32, 4, 250, 450, 0.1e6,
                          400e6, seed, interval=100)]


CONFIG4_GRIDS = [(16, 4), (12, 4), (8, 4), (16, 2), (6, 4), (12, 2), (8, 2), (4, 4)]


def feasible_periodic_length(confined, nmol, wall):
    """Shortest periodic length of the liquid-density lattice start (A)."""
    if confined == 0:
        return math.ceil(nmol ** (1.0 / 3.0) - 1e-9) * 3.1
    if confined == 1:
        racc = max(wall - 2.6, 0.0)
        m = int(racc // 2.9)
        k = sum(1 for i in range(-m, m + 1) for j in range(-m, m + 1)
                if (i * 2.9) ** 2 + (j * 2.9) ** 2 <= racc ** 2 + 1e-9)
        return math.ceil(nmol / k) * 3.0
    zacc = max(wall / 2.0 - 1.8, 0.0)
    nz = int(2 * zacc // 2.9) + 1
    return math.ceil(math.sqrt(nmol / nz)) * 3.1


def feasible_geometry(rng, confined, nmol, tube_r, slit_w, rc):
    """(confined, wall, rc) for a drawn system: a liquid-density lattice whose
    periodic length would fall below 2*rc+2 A (the minimum-image bound) gets the
    largest feasible rc >= 8.5 A; if none exists the system becomes a nanotube,
    whose periodic length grows with nmol (rc redrawn, radius shrunk until it fits)."""
    wall = tube_r if confined == 1 else slit_w if confined == 2 else 0.0
    Lp = feasible_periodic_length(confined, nmol, wall)
    if Lp < 2.0 * rc + 2.0:
        rc = (Lp - 2.0) / 2.0
        if rc < 8.5:
            confined, wall, rc = 1, tube_r, float(rng.uniform(8.5, 12.0))
            while feasible_periodic_length(1, nmol, wall) < 2.0 * rc + 2.0:
                wall -= 0.25
    return confined, wall, rc


def config4(seed=4, interval=100):
    """8 ensembles, 256 replicas: nmol log-uniform 64-2048, models uniform over
    TIP3P/4P/5P, confinement uniform over bulk/tube (R 6-8 A)/slit (7-14 A),
    rc 8.5-12 (rs = rc-1 or rc-2), grids over 200-400 K x 0.1-300 MPa.

    A drawn (confinement, rc) whose liquid-density lattice would have a
    periodic length below 2*rc+2 A (the minimum-image bound) gets the largest
    feasible rc >= 8.5 A; if none exists the system becomes a nanotube, whose
    periodic length grows with nmol.  So no system is inflated to gas density."""
    rng = np.random.default_rng(seed)
    grids = [CONFIG4_GRIDS[i] for i in rng.permutation(len(CONFIG4_GRIDS))]
    out = []
    for e, (nt, npr) in enumerate(grids):
        nmol = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        model = ["tip3p", "tip4p", "tip5p"][rng.integers(3)]
        confined = int(rng.integers(3))
        # radii below ~6 A leave room for a single file of molecules only, whose
        # thermostat variable drifts far faster than in any other geometry here
        tube_r = float(rng.uniform(6.0, 8.0))
        slit_w = float(rng.uniform(7.0, 14.0))
        rc = float(rng.uniform(8.5, 12.0))
        drs = float(rng.choice([1.0, 2.0]))
        confined, wall, rc = feasible_geometry(rng, confined, nmol, tube_r, slit_w, rc)
        out.append(make_ensemble(f"config4.{e}", model, confined, nmol, wall, rc, rc - drs, nt,
                                 npr, 200, 400, 0.1e6, 300e6, seed * 1000 + e, interval=interval))
    return out


SERVING_RATE = 20.0   # mean job arrivals per second


def config5_arrivals(seed=5, njobs=8, rate=SERVING_RATE):
    """Poisson arrival times (s) of the serving stream."""
    rng = np.random.default_rng([seed, 1 << 20])
    return np.cumsum(rng.exponential(1.0 / rate, njobs))


def config5_job(seed, k, interval=100):
    """Job k of the serving stream: nmol log-uniform 96-4096, model uniform over
    TIP3P/4P/5P, confinement uniform over bulk/tube (R 6-8 A)/slit (7-14 A), rc
    8.5-12 (rs = rc-1 or rc-2), 8-64 replicas (npress 1/2/4) over 200-400 K x
    0.1-300 MPa, interval 100, ninterval 10-200.  Returns (ensemble, ninterval)."""
    rng = np.random.default_rng([seed, k])
    nmol = int(round(math.exp(rng.uniform(math.log(96), math.log(4096)))))
    model = ["tip3p", "tip4p", "tip5p"][rng.integers(3)]
    confined = int(rng.integers(3))
    tube_r = float(rng.uniform(6.0, 8.0))
    slit_w = float(rng.uniform(7.0, 14.0))
    rc = float(rng.uniform(8.5, 12.0))
    drs = float(rng.choice([1.0, 2.0]))
    npr = int([1, 2, 4][rng.integers(3)])
    nt = int(rng.integers(-(-8 // npr), 64 // npr + 1))
    ninterval = int(rng.integers(10, 201))
    confined, wall, rc = feasible_geometry(rng, confined, nmol, tube_r, slit_w, rc)
    ens = make_ensemble(f"config5.{k}", model, confined, nmol, wall, rc, rc - drs, nt, npr, 200,
                        400, 0.1e6, 300e6, seed * 1000 + k, interval=interval)
    return ens, ninterval


def small_ensemble(model="tip4p", confined=0, nmol=64, ntemp=2, npress=2, seed=11,
                   rc=8.5, rs=7.5, wall=None, interval=10, nfwall=1000, pconstant=None,
                   tconstant=1):
    """A small test system (seconds for the FP64 oracle)."""
    if wall is None:
        wall = {0: 0.0, 1: 6.0, 2: 10.0}[confined]
    return make_ensemble(f"small.{model}.{confined}", model, confined, nmol, wall, rc, rs, ntemp,
                         npress, 250, 350, 0.1e6, 200e6, seed, nfwall=nfwall, interval=interval,
                         pconstant=pconstant, tconstant=tconstant)
