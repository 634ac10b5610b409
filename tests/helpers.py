"""Input generators and coordinate helpers shared by the tests."""
import numpy as np


def seeded_ics(n, seed, planar=False, r_range=(0.5, 2.0), log_r=False):
    """Config-0 style initial conditions (R, vR, vT, z, vz, phi)."""
    rng = np.random.default_rng(seed)
    if log_r:
        R = np.exp(rng.uniform(np.log(r_range[0]), np.log(r_range[1]), n))
    else:
        R = rng.uniform(r_range[0], r_range[1], n)
    vR = rng.normal(0, 0.1, n)
    vT = 1 + rng.normal(0, 0.1, n)
    z = rng.normal(0, 0.05, n)
    vz = rng.normal(0, 0.05, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    if planar:
        return np.stack([R, vR, vT, phi], 1)
    return np.stack([R, vR, vT, z, vz, phi], 1)


def cyl_to_rect(v):
    """galpy's cyl_to_rect_galpy / polar_to_rect_galpy on rows."""
    v = np.asarray(v)
    if v.shape[-1] == 4:
        R, vR, vT, phi = (v[..., k] for k in range(4))
        c, s = np.cos(phi), np.sin(phi)
        return np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c], -1)
    R, vR, vT, z, vz, phi = (v[..., k] for k in range(6))
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz], -1)


def rect_to_cyl(o):
    o = np.asarray(o)
    if o.shape[-1] == 4:
        x, y, vx, vy = (o[..., k] for k in range(4))
        phi = np.arctan2(y, x)
        c, s = np.cos(phi), np.sin(phi)
        return np.stack([np.hypot(x, y), vx * c + vy * s, -vx * s + vy * c, phi], -1)
    x, y, z, vx, vy, vz = (o[..., k] for k in range(6))
    phi = np.arctan2(y, x)
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([np.hypot(x, y), vx * c + vy * s, -vx * s + vy * c, z, vz, phi], -1)


def cyl_diff(a, b):
    """|a-b| on cylindrical rows with the angle compared modulo 2 pi."""
    d = np.abs(np.asarray(a) - np.asarray(b))
    k = a.shape[-1] - 1
    d[..., k] = np.abs((a[..., k] - b[..., k] + np.pi) % (2 * np.pi) - np.pi)
    return d


def unit_deviations(w_base, dim):
    """One row per canonical deviation direction of each base orbit."""
    n = len(w_base)
    nv = 2 * dim
    w = np.zeros((n * nv, 2 * nv))
    for i in range(n):
        for j in range(nv):
            w[i * nv + j, :nv] = w_base[i]
            w[i * nv + j, nv + j] = 1.0
    return w


# differentiable parameters per component type and their galpy argument index
ADJ_PARAM_ARGS = {15: (0, 2), 5: (0, 1, 2), 9: (0, 1), 8: (0, 1), 0: (0, 1, 2)}


def galpy_nargs(t, planar):
    return {15: 3 if planar else 5, 5: 3, 9: 2, 8: 2, 0: 4}[int(t)]


def adj_param_index(pot_type, planar):
    """pot_args index of every differentiable parameter, in the adjoint's order."""
    idx, off = [], 0
    for t in pot_type:
        idx += [off + a for a in ADJ_PARAM_ARGS[int(t)]]
        off += galpy_nargs(t, planar)
    return np.array(idx, dtype=np.int64)


def central_fd(f, x, idx, rel=1e-6, floor=1e-3):
    """Central differences of f (array-valued) with respect to x[idx], with
    steps rel * max(|x|, floor); returns [len(idx), *f.shape]."""
    out = []
    for j in idx:
        h = rel * max(abs(x[j]), floor)
        xp, xm = x.copy(), x.copy()
        xp[j] += h
        xm[j] -= h
        out.append((f(xp) - f(xm)) / (2 * h))
    return np.array(out)


def differentiation_workload(n, seed=3):
    """Planar MWPotential2014 gradient workload: config-0 style initial
    conditions in the plane (z = vz = 0) as rectangular (x, y, vx, vy), and
    seeded targets of the same shape for L = sum |y(20) - target|^2."""
    w0 = cyl_to_rect(seeded_ics(n, seed, planar=True))
    tgt = cyl_to_rect(seeded_ics(n, seed + 100, planar=True))
    return np.ascontiguousarray(w0), np.ascontiguousarray(tgt)


# the spherical and axisymmetric (FlattenedPower, KuzminKutuzovStaeckel)
# potentials added behind the component template (golden-vector names)
ADDED_POTS = ["power", "kepler", "jaffe", "isochrone", "plummer", "pseudoiso", "burkert",
             "dehnencore", "dehnen", "homsphere", "null", "einasto", "exptruncnfw",
              "flatpower", "flatlog", "kks", "kuzmindisk"]
# forces with a kink (the homogeneous sphere's surface) or a jump (the
# Kuzmin disk's plane): an adaptive step whose stages straddle it can be
# accepted on one side of a rounding difference and rejected on the other,
# and dopr54 forces its smallest step there (err = 1, as the reference)
KINKED = ("homsphere", "kuzmindisk")


def golden_pot(golden, name, planar=False):
    """(pot_type, pot_args) of a golden potential as galpy parses it (the
    planar argument list where the golden file holds one)."""
    if planar and f"{name}_planar_args" in golden:
        return golden[f"{name}_planar_type"], golden[f"{name}_planar_args"]
    return golden[f"{name}_type"], golden[f"{name}_args"]


def cyl_to_sos(v):
    """galpy's cyl_to_sos_galpy on rows (R, vR, vT, z, vz, phi, t) ->
    (x, y, vx, vy, A, t, psi)."""
    v = np.asarray(v, dtype=float)
    R, vR, vT, z, vz, phi, t = (v[..., k] for k in range(7))
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c, np.sqrt(z * z + vz * vz),
                     t, np.arctan2(z, vz)], -1)


def sos_to_cyl(v):
    """galpy's sos_to_cyl_galpy on rows (x, y, vx, vy, A, t, psi) ->
    (R, vR, vT, z, vz, phi, t)."""
    v = np.asarray(v, dtype=float)
    x, y, vx, vy, A, t, psi = (v[..., k] for k in range(7))
    phi = np.arctan2(y, x)
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([np.sqrt(x * x + y * y), vx * c + vy * s, -vx * s + vy * c, A * np.sin(psi),
                     A * np.cos(psi), phi, t], -1)


def sos_diff(a, b):
    """Elementwise |a - b| of (R, vR, vT, z, vz, phi, t) rows, phi wrapped."""
    d = np.abs(np.asarray(a) - np.asarray(b))
    d[..., 5] = np.abs((a[..., 5] - b[..., 5] + np.pi) % (2 * np.pi) - np.pi)
    return d


def polar_to_sos(v, surface):
    """galpy's polar_to_sos_galpy on rows (R, vR, vT, phi, t): surface 1
    (y = 0) -> (x, vx, A, t, psi), otherwise (x = 0) -> (y, vy, A, t, psi)."""
    v = np.asarray(v, dtype=float)
    R, vR, vT, phi, t = (v[..., k] for k in range(5))
    c, s = np.cos(phi), np.sin(phi)
    x, y, vx, vy = R * c, R * s, vR * c - vT * s, vR * s + vT * c
    if surface == 1:
        return np.stack([x, vx, np.sqrt(y * y + vy * vy), t, np.arctan2(y, vy)], -1)
    return np.stack([y, vy, np.sqrt(x * x + vx * vx), t, np.arctan2(x, vx)], -1)


def sos_to_polar(v, surface):
    """galpy's sos_to_polar_galpy on rows -> (R, vR, vT, phi, t)."""
    v = np.asarray(v, dtype=float)
    u, vu, A, t, psi = (v[..., k] for k in range(5))
    w, vw = A * np.sin(psi), A * np.cos(psi)
    x, vx, y, vy = (u, vu, w, vw) if surface == 1 else (w, vw, u, vu)
    phi = np.arctan2(y, x)
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([np.sqrt(x * x + y * y), vx * c + vy * s, -vx * s + vy * c, phi, t], -1)
