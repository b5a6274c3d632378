"""Independent numpy statement of the perturbative vacuum expectation values twvev
computes (Q/vevbleft.f90:757-2536), used to check the oracle's literal restatement.

Instead of the reference's site-by-site shell enumeration, the hopping expansion is
taken on the full lattice: for a unit source e(x, colour, spin),
    sb_n = (D R)^n (cos(delta) e),
    (D v)(y) = sum_mu U_mu(y) (r - gamma_mu) v(y + mu) + U_mu(y - mu)^+ (r + gamma_mu) v(y - mu),
    R = cos(delta) - sin(delta) J,  (J v) = (v_3, v_4, -v_1, -v_2)  (spins 1..4),
periodic in space and time without a boundary sign; dobndry = 1 drops the time hops
across the last slice.  Where no two unwrapped offsets of the reference's shells meet
on the lattice (every extent >= 8), the reference's orders equal these full-lattice
powers at every site it reads, so the two statements must agree.

The operators are written in closed form with S = xk1 R sb1 + xk3 R sb3 (or xk3 R sb3
without twist; xk5 R sb5 for the second level), T = xk2 R sb2 + xk4 R sb4 (xk4 R sb4;
xk6 R sb6), xk(n) = (kappa cos(delta))^n, source spin d, colour c:
    rho(x)       = cA(d) sum_b S(x+t)[d, b] U_t(x)[c, b]
    rho(x-t)     = cL(d) sum_b S(x-t)[d, b] conj(U_t(x-t)[b, c])
    J_mu(x)      = sum_b (-r S(x+mu)[d, b] + ph_mu(d) S(x+mu)[o_mu(d), b]) U_mu(x)[c, b]
    J_mu(x-mu)   = sum_b ( r S(x-mu)[d, b] + ph_mu(d) S(x-mu)[o_mu(d), b]) conj(U_mu(x-mu)[b, c])
    psibar psi   = T[d, c],   psibar g5 psi = -i sgn(d) T[cd(d), c]
with cL = r + g4(d), cA = -(r - g4(d)), g4 = (1, 1, -1, -1), o_1 = o_2 = 5 - d,
o_3 = (3, 4, 1, 2), ph_1 = 1, ph_2 = -i (d odd) / i (d even), ph_3 = 1 (d odd) / -1
(d even), cd = (3, 4, 1, 2), sgn = (1, 1, -1, -1).
"""
import numpy as np

# gamma matrices of the expansion (the reference's basis, spins 0-based)
GAM = [np.zeros((4, 4), complex) for _ in range(4)]
for j in range(4):
    GAM[0][j, 3 - j] = 1.0
GAM[1][0, 3], GAM[1][1, 2], GAM[1][2, 1], GAM[1][3, 0] = -1j, 1j, -1j, 1j
GAM[2][0, 2], GAM[2][1, 3], GAM[2][2, 0], GAM[2][3, 1] = 1.0, -1.0, 1.0, -1.0
GAM[3] = np.diag([1.0, 1.0, -1.0, -1.0]).astype(complex)
AXIS = (3, 2, 1, 0)  # mu -> axis of a (nt, nz, ny, nx, ...) array


def rotation(delta):
    c, s = np.cos(delta), np.sin(delta)
    R = np.zeros((4, 4))
    R[0, 0] = R[1, 1] = R[2, 2] = R[3, 3] = c
    R[0, 2] = R[1, 3] = -s
    R[2, 0] = R[3, 1] = s
    return R


def spin(P, v):
    return np.einsum("st,...tb->...sb", P, v)


def hop(links, v, r, fixbc):
    out = np.zeros_like(v)
    eye = np.eye(4)
    for mu in range(4):
        ax, U = AXIS[mu], links[mu]
        t1 = np.einsum("...ab,...sb->...sa", U, spin(r * eye - GAM[mu], np.roll(v, -1, axis=ax)))
        t2 = np.einsum("...ba,...sb->...sa", np.roll(U, 1, axis=ax).conj(),
                       spin(r * eye + GAM[mu], np.roll(v, 1, axis=ax)))
        if mu == 3 and fixbc:
            t1[-1] = 0.0
            t2[0] = 0.0
        out += t1 + t2
    return out


def momentum_factors(dims, io):
    """ffac, fas1, fas2, fas3 [k = 1..4] at spatial site (x, y, z) 0-based."""
    nx, ny, nz, _ = dims
    p1, p2, p3 = 8.0 * np.arctan(1.0) / nx, 8.0 * np.arctan(1.0) / ny, 8.0 * np.arctan(1.0) / nz

    def f(x, y, z):
        dx, dy, dz = (x + 1 - io[0]) * p1, (y + 1 - io[1]) * p2, (z + 1 - io[2]) * p3
        cx, cy, cz, sx, sy, sz = np.cos(dx), np.cos(dy), np.cos(dz), np.sin(dx), np.sin(dy), np.sin(dz)
        ffac = [None, (cx + cy + cz) / 3, (cx * cy + cx * cz + cy * cz) / 3, cx * cy * cz,
                (np.cos(2 * dx) + np.cos(2 * dy) + np.cos(2 * dz)) / 3]
        fas1 = [None, sx, sx * (cy + cz) / 2, sx * cy * cz, np.sin(2 * dx)]
        fas2 = [None, sy, sy * (cx + cz) / 2, sy * cx * cz, np.sin(2 * dy)]
        fas3 = [None, sz, sz * (cx + cy) / 2, sz * cx * cy, np.sin(2 * dz)]
        return ffac, fas1, fas2, fas3

    return f


def twvev_sites(links, dims, sites, kappa, delta=0.0, io=(1, 1, 1), dobndry=0, r=1):
    """opertemp contributions (isb, ix, t, op) of the listed 1-based lexicographic sites."""
    nx, ny, nz, nt = dims
    fixbc = dobndry == 1
    R = rotation(delta)
    c = np.cos(delta)
    xk = [(kappa * c) ** n for n in range(7)]
    twist = abs(delta) > 1e-12
    mf = momentum_factors(dims, io)
    O = np.zeros((2, 5, nt, 12))
    g4 = (1, 1, -1, -1)
    o3 = (2, 3, 0, 1)
    cdm = (2, 3, 0, 1)
    sgn = (1, 1, -1, -1)
    for site in sites:
        L = site - 1
        x = [L % nx, (L // nx) % ny, (L // (nx * ny)) % nz, L // (nx * ny * nz)]
        pos = (x[3], x[2], x[1], x[0])

        def shifted(mu, s):
            p = list(x)
            p[mu] = (p[mu] + s) % dims[mu]
            return (p[3], p[2], p[1], p[0])

        for d in range(4):
            for col in range(3):
                e = np.zeros((nt, nz, ny, nx, 4, 3), complex)
                e[pos][d, col] = c
                sb, cur = [None], e
                for _ in range(6):
                    cur = hop(links, spin(R, cur), r, fixbc)
                    sb.append(spin(R, cur))
                for isb in range(2):
                    if isb == 0:
                        S = xk[1] * sb[1] + xk[3] * sb[3] if twist else xk[3] * sb[3]
                        T = (xk[2] * sb[2] + xk[4] * sb[4] if twist else xk[4] * sb[4])[pos]
                    else:
                        S, T = xk[5] * sb[5], (xk[6] * sb[6])[pos]
                    Ut = links[3]
                    rho_x = -(r - g4[d]) * np.sum(S[shifted(3, 1)][d, :] * Ut[pos][col, :])
                    rho_l = (r + g4[d]) * np.sum(S[shifted(3, -1)][d, :] * Ut[shifted(3, -1)][:, col].conj())
                    if fixbc and x[3] == nt - 1:
                        rho_x = 0.0
                    if fixbc and x[3] == 0:
                        rho_l = 0.0
                    J, Jl = [None] * 3, [None] * 3
                    for mu in range(3):
                        od = 3 - d if mu < 2 else o3[d]
                        if mu == 0:
                            ph = 1.0
                        elif mu == 1:
                            ph = -1j if d % 2 == 0 else 1j
                        else:
                            ph = 1.0 if d % 2 == 0 else -1.0
                        U = links[mu]
                        Sp, Sm = S[shifted(mu, 1)], S[shifted(mu, -1)]
                        J[mu] = np.sum((-r * Sp[d, :] + ph * Sp[od, :]) * U[pos][col, :])
                        Jl[mu] = np.sum((r * Sm[d, :] + ph * Sm[od, :]) * U[shifted(mu, -1)][:, col].conj())
                    psi = T[d, col]
                    psu = -1j * sgn[d] * T[cdm[d], col]
                    t, tm = x[3], (x[3] - 1) % nt
                    o = O[isb]
                    o[0, t, 0] += rho_x.real
                    o[0, t, 1] += rho_x.imag
                    o[0, tm, 0] += rho_l.real
                    o[0, tm, 1] += rho_l.imag
                    o[0, t, 2] += psi.real
                    o[0, t, 3] += psi.imag
                    for mu in range(3):
                        v = J[mu] + Jl[mu]
                        o[0, t, 4 + 2 * mu] += v.real
                        o[0, t, 5 + 2 * mu] += v.imag
                    o[0, t, 10] += psu.real
                    o[0, t, 11] += psu.imag
                    here = mf(x[0], x[1], x[2])
                    lx = mf((x[0] - 1) % nx, x[1], x[2])
                    ly = mf(x[0], (x[1] - 1) % ny, x[2])
                    lz = mf(x[0], x[1], (x[2] - 1) % nz)
                    for k in range(1, 5):
                        ff = here[0][k]
                        o[k, t, 0] += rho_x.real * ff
                        o[k, t, 1] += rho_x.imag * ff
                        o[k, tm, 0] += rho_l.real * ff
                        o[k, tm, 1] += rho_l.imag * ff
                        o[k, t, 2] += psi.real * ff
                        o[k, t, 3] += psi.imag * ff
                        o[k, t, 4] += J[0].imag * here[3][k] + Jl[0].imag * lx[3][k]
                        o[k, t, 5] += J[1].imag * here[1][k] + Jl[1].imag * ly[1][k]
                        o[k, t, 6] += J[2].imag * here[2][k] + Jl[2].imag * lz[2][k]
                        o[k, t, 7] += J[0].imag * here[2][k] + Jl[0].imag * lx[2][k]
                        o[k, t, 8] += J[1].imag * here[3][k] + Jl[1].imag * ly[3][k]
                        o[k, t, 9] += J[2].imag * here[1][k] + Jl[2].imag * lz[1][k]
                        o[k, t, 10] += psu.real * ff
                        o[k, t, 11] += psu.imag * ff
    return O
