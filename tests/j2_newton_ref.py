"""Dense Newton on the oracle's J2 restatement (test infrastructure): the reference answer for the
quasi-static J2 load path tests."""
import numpy as np


def top_shear_load(spec, eqmap, total):
    """x-direction nodal loads of a uniform shear traction on the top face summing to `total`."""
    nx, ny, nz, hx, hy, _ = spec.grid
    ci = np.full(nx + 1, 2.0)
    cj = np.full(ny + 1, 2.0)
    ci[[0, -1]] = 1.0
    cj[[0, -1]] = 1.0
    i, j = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    tags = 1 + i + (nx + 1) * (j + (ny + 1) * nz)
    share = total / (4.0 * nx * ny)
    q = eqmap[tags.ravel(), 0]
    f = np.zeros(int(eqmap.max()) + 1)
    np.add.at(f, q[q >= 0], (share * np.outer(ci, cj)).ravel()[q >= 0])
    return f, int(eqmap[tags[-1, -1], 0])


def dense_newton_path(pm, fext_unit, factors, monitor, tol=1e-6, max_newton=30):
    """The load path with NormUnbalance ||f_ext - f_int|| <= tol (absolute), direct solves."""
    n = len(fext_unit)
    committed = pm.j2_state()
    u = np.zeros(n)
    zero = np.zeros(n)
    out, plastic = [], []
    for lam in factors:
        fext = lam * fext_unit
        for it in range(max_newton + 1):
            f, trial, D, npl = pm.force_j2(committed, u, zero)
            r = fext - f
            if np.linalg.norm(r) <= tol:
                break
            assert it < max_newton, "oracle Newton did not converge"
            K = np.stack([pm.apply_j2(D, (1.0, 0.0, 0.0), e) for e in np.eye(n)], axis=1)
            u = u + np.linalg.solve(K, r)
        committed = trial
        out.append(u[monitor])
        plastic.append(npl)
    return np.array(out), np.array(plastic)


def dense_newmark(pm, load, steps, dt, monitor, lumped_mass=None, beta=0.25, gamma=0.5, tol=1e-6, max_newton=30):
    """Newmark steps (Newmark::newStep with displ == 1, the stage's Newton loop with inertia) on the
    oracle's elastic operator with direct solves: the reference answer for the transient tests.
    M a is lumped_mass * a when given, else the oracle's mass operator."""
    n = pm.n
    c2, c3 = gamma / (beta * dt), 1.0 / (beta * dt * dt)
    a1, a2, a3, a4 = 1.0 - gamma / beta, dt * (1.0 - 0.5 * gamma / beta), -1.0 / (beta * dt), 1.0 - 0.5 / beta
    K = np.stack([pm.apply_operator((1.0, c2, c3), e) for e in np.eye(n)], axis=1)
    u, v, a = np.zeros(n), np.zeros(n), np.zeros(n)
    out = []
    for i in range(steps):
        vt, at = v.copy(), a.copy()
        v = v * a1 + at * a2
        a = a * a4 + vt * a3
        fext = load((i + 1) * dt)
        for it in range(max_newton + 1):
            ma = lumped_mass * a if lumped_mass is not None else pm.apply_operator((0.0, 0.0, 1.0), a)
            r = fext - pm.force(u, v) - ma
            if np.linalg.norm(r) <= tol:
                break
            assert it < max_newton, "oracle Newmark did not converge"
            du = np.linalg.solve(K, r)
            u, v, a = u + du, v + c2 * du, a + c3 * du
        out.append(u[monitor])
    return np.array(out)
