"""CPU restatement (NumPy, FP64) of the reference's MMA subproblem: ``mma.mmasub`` and
``mma.subsolv`` (sttopt/mma.py:150-557, Svanberg's method of moving asymptotes with a
primal-dual interior-point Newton solve of the separable subproblem).

Test infrastructure only, like ``sttopt_oracle``: the tests use it as the checker of the
device ``sttopt_b200.mma`` and pin it to the reference's own outputs
(``tests/golden/mma.npz``).  The line search tries one halving at a time
(sttopt/mma.py:297-343, ``chunks=None``), which the chunked search equals by construction.
"""

from __future__ import annotations

import numpy as np

EPSIMIN = 1e-7  # sttopt/mma.py:218
MAX_HALVINGS = 50  # sttopt/mma.py:289
MAX_NEWTON = 200  # sttopt/mma.py:442


def asymptotes(iteration, xval, xmin, xmax, xold1, xold2, low, upp, asyinit, asyclamp_min, asyclamp_max,
               asyincr, asydecr):
    """The moving asymptotes (sttopt/mma.py:226-247): from scratch on the first two
    iterations, else widened where x moved monotonically and narrowed where it
    oscillated, clamped to [asyclamp_min, asyclamp_max] times the range."""
    xrange = xmax - xmin
    if iteration < 2:
        return xval - asyinit * xrange, xval + asyinit * xrange
    zzz = (xval - xold1) * (xold1 - xold2)
    factor = np.where(zzz > 0, asyincr, np.where(zzz < 0, asydecr, 1.0))
    low = xval - factor * (xold1 - low)
    upp = xval + factor * (upp - xold1)
    low = np.minimum(np.maximum(low, xval - asyclamp_max * xrange), xval - asyclamp_min * xrange)
    upp = np.maximum(np.minimum(upp, xval + asyclamp_max * xrange), xval + asyclamp_min * xrange)
    return low, upp


def approximation(xval, xmin, xmax, low, upp, df0dx, fval, dfdx, move, raa0, albefa):
    """Move limits alfa, beta and the separable approximation p0, q0, P, Q, b
    (sttopt/mma.py:249-285)."""
    xrange = xmax - xmin
    alfa = np.maximum(np.maximum(low + albefa * (xval - low), xval - move * xrange), xmin)
    beta = np.minimum(np.minimum(upp - albefa * (upp - xval), xval + move * xrange), xmax)
    xmamiinv = 1.0 / np.maximum(xrange, 1e-5)
    ux1, xl1 = upp - xval, xval - low
    ux2, xl2 = ux1 * ux1, xl1 * xl1
    p0, q0 = np.maximum(df0dx, 0.0), np.maximum(-df0dx, 0.0)
    pq0 = 0.001 * (p0 + q0) + raa0 * xmamiinv
    p0, q0 = (p0 + pq0) * ux2, (q0 + pq0) * xl2
    P, Q = np.maximum(dfdx, 0.0), np.maximum(-dfdx, 0.0)
    PQ = 0.001 * (P + Q) + raa0 * xmamiinv[None, :]
    P, Q = (P + PQ) * ux2[None, :], (Q + PQ) * xl2[None, :]
    b = P @ (1.0 / ux1) + Q @ (1.0 / xl1) - fval
    return alfa, beta, p0, q0, P, Q, b


def mmasub(m, n, iteration, xval, xmin, xmax, xold1, xold2, f0val, df0dx, fval, dfdx, low, upp, a0, a, c, d,
           asyinit=0.5, asyclamp_min=0.01, asyclamp_max=10.0, move=0.5, raa0=1e-5, albefa=0.1, asyincr=1.2,
           asydecr=0.7, stats=None):
    """One MMA step (sttopt/mma.py:150-285): ``(xmma, ymma, zmma, lam, xsi, eta, mu, zet, s,
    low, upp)``; ``stats`` as in ``subsolv``."""
    low, upp = asymptotes(iteration, xval, xmin, xmax, xold1, xold2, low, upp, asyinit, asyclamp_min,
                          asyclamp_max, asyincr, asydecr)
    alfa, beta, p0, q0, P, Q, b = approximation(xval, xmin, xmax, low, upp, df0dx, fval, dfdx, move, raa0,
                                                albefa)
    return subsolv(m, n, EPSIMIN, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d, stats) + (low, upp)


def _residual(pt, epsi, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d):
    """The KKT residual of the barrier problem at a point (sttopt/mma.py:399-434), in the
    reference's order: rex, rey, rez, relam, rexsi, reeta, remu, rezet, res."""
    x, y, z, lam, xsi, eta, mu, zet, s = pt
    ux1, xl1 = upp - x, x - low
    plam, qlam = p0 + lam @ P, q0 + lam @ Q
    gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
    rex = plam / (ux1 * ux1) - qlam / (xl1 * xl1) - xsi + eta
    rey = c + d * y - mu - lam
    rez = a0 - zet - lam @ a
    relam = gvec - a * z - y + s - b
    return np.concatenate([rex, rey, [rez], relam, xsi * (x - alfa) - epsi, eta * (beta - x) - epsi,
                           mu * y - epsi, [zet * z - epsi], lam * s - epsi])


def subsolv(m, n, epsimin, low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d, stats=None):
    """The subproblem's primal-dual Newton solve along the barrier path epsi = 1, 0.1, ...
    (sttopt/mma.py:346-557): both eliminations of the bordered KKT system (m < n and
    m >= n), the fraction-to-the-boundary step limit and the residual-norm line search.
    ``stats`` (a dict) gathers the levels stopped at the Newton cap as the reference does
    (``subsolv_cap_hits``), and the Newton steps and line-search candidates tried
    (``subsolv_newton_steps``, ``subsolv_line_search_tries``)."""
    counts = {"subsolv_cap_hits": 0, "subsolv_newton_steps": 0, "subsolv_line_search_tries": 0}
    x = 0.5 * (alfa + beta)
    y, z, lam = np.ones(m), 1.0, np.ones(m)
    xsi = np.maximum(1.0 / (x - alfa), 1.0)
    eta = np.maximum(1.0 / (beta - x), 1.0)
    mu = np.maximum(np.ones(m), 0.5 * c)
    zet, s = 1.0, np.ones(m)
    epsi = 1.0
    args = (low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d)
    while epsi > epsimin:
        residu = _residual((x, y, z, lam, xsi, eta, mu, zet, s), epsi, *args)
        residunorm = np.linalg.norm(residu)
        residumax = np.abs(residu).max()
        ittt = 0
        while residumax > 0.9 * epsi and ittt < MAX_NEWTON:
            ittt += 1
            counts["subsolv_newton_steps"] += 1
            ux1, xl1 = upp - x, x - low
            ux2, xl2 = ux1 * ux1, xl1 * xl1
            ux3, xl3 = ux1 * ux2, xl1 * xl2
            plam, qlam = p0 + P.T @ lam, q0 + Q.T @ lam
            gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
            GG = P * (1.0 / ux2)[None, :] - Q * (1.0 / xl2)[None, :]
            delx = plam / ux2 - qlam / xl2 - epsi / (x - alfa) + epsi / (beta - x)
            dely = c + d * y - lam - epsi / y
            delz = a0 - a @ lam - epsi / z
            dellam = gvec - a * z - y - b + epsi / lam
            diagx = 2 * (plam / ux3 + qlam / xl3) + xsi / (x - alfa) + eta / (beta - x)
            diagy = d + mu / y
            diaglamyi = s / lam + 1.0 / diagy
            if m < n:
                blam = dellam + dely / diagy - GG @ (delx / diagx)
                Alam = np.diag(diaglamyi) + (GG * (1.0 / diagx)[None, :]) @ GG.T
                AA = np.block([[Alam, a[:, None]], [a[None, :], np.array([[-zet / z]])]])
                solut = np.linalg.solve(AA, np.concatenate([blam, [delz]]))
                dlam, dz = solut[:m], solut[m]
                dx = -delx / diagx - (GG.T @ dlam) / diagx
            else:
                dellamyi = dellam + dely / diagy
                Axx = np.diag(diagx) + (GG.T * (1.0 / diaglamyi)[None, :]) @ GG
                azz = zet / z + a @ (a / diaglamyi)
                axz = -GG.T @ (a / diaglamyi)
                bx = delx + GG.T @ (dellamyi / diaglamyi)
                bz = delz - a @ (dellamyi / diaglamyi)
                AA = np.block([[Axx, axz[:, None]], [axz[None, :], np.array([[azz]])]])
                solut = np.linalg.solve(AA, np.concatenate([-bx, [-bz]]))
                dx, dz = solut[:n], solut[n]
                dlam = (GG @ dx) / diaglamyi - dz * (a / diaglamyi) + dellamyi / diaglamyi
            dy = -dely / diagy + dlam / diagy
            dxsi = -xsi + epsi / (x - alfa) - (xsi * dx) / (x - alfa)
            deta = -eta + epsi / (beta - x) + (eta * dx) / (beta - x)
            dmu = -mu + epsi / y - (mu * dy) / y
            dzet = -zet + epsi / z - zet * dz / z
            ds = -s + epsi / lam - (s * dlam) / lam
            xx = np.concatenate([y, [z], lam, xsi, eta, mu, [zet], s])
            dxx = np.concatenate([dy, [dz], dlam, dxsi, deta, dmu, [dzet], ds])
            steg = 1.0 / max((-1.01 * dx / (x - alfa)).max(), (1.01 * dx / (beta - x)).max(),
                             (-1.01 * dxx / xx).max(), 1.0)
            old = (x, y, z, lam, xsi, eta, mu, zet, s)
            dirs = (dx, dy, dz, dlam, dxsi, deta, dmu, dzet, ds)
            for j in range(MAX_HALVINGS):
                counts["subsolv_line_search_tries"] += 1
                t = steg / 2.0 ** j
                pt = tuple(o + t * dv for o, dv in zip(old, dirs))
                residu = _residual(pt, epsi, *args)
                resinew = np.linalg.norm(residu)
                if not resinew > residunorm:  # a NaN norm is accepted, as in the reference
                    break
            x, y, z, lam, xsi, eta, mu, zet, s = pt
            residunorm, residumax = resinew, np.abs(residu).max()
        if ittt > MAX_NEWTON - 2:  # sttopt/mma.py:540
            counts["subsolv_cap_hits"] += 1
        epsi = 0.1 * epsi
    if stats is not None:
        for k, v in counts.items():
            stats[k] = stats.get(k, 0) + v
    return x, y, z, lam, xsi, eta, mu, zet, s
