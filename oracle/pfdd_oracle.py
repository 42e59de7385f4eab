"""CPU oracle: a numpy restatement of the reference PFDD Ginzburg-Landau step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module;
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
it, and only as the checker.

Every function cites the reference file:line it restates (paths inside the
reference project's src/).  Semantics kept exactly, including the reference's
quirks:
  * the state xi is complex and the FFTs are full 3-D complex-to-complex,
    unnormalised both ways, 1/N applied in the update (fft_fftw_slab.cpp:1773);
  * B(k) uses the frequency convention of frec() (k_i in [-1/2, 1/2), index
    n/2 maps to -1/2), so B at index -k differs from B at k on the Nyquist
    planes and a real xi grows an imaginary part there;
  * core_energy_sine scales isf before using it in Cn
    (fft_fftw_slab.cpp:1403-1404);
  * core_energy_pyrII writes dE_core only at the last site of each system
    (fft_fftw_slab.cpp:1491);
  * update_order_parameter accumulates xinorm with a stale previous value on
    masked sites (fft_fftw_slab.cpp:1769-1781).

Parity pin: tests/test_oracle_vs_reference.py runs this module and the
reference sources compiled in oracle/_ref (built by oracle/ref_build/Makefile)
on the same decks and states; tests/golden/ holds fixtures written by the
compiled reference (tests/golden/make_golden.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI = math.pi


# ---------------------------------------------------------------- elasticity
def stiffness(C44: float, C12: float) -> np.ndarray:
    """Isotropic C_ijkm (fft_fftw_slab.cpp:373-391)."""
    d = np.eye(3)
    return (C44 * (np.einsum("ik,jm->ijkm", d, d) + np.einsum("im,jk->ijkm", d, d))
            + C12 * np.einsum("ij,km->ijkm", d, d))


def voigt_constants(C44: float, C12: float, C11: float):
    """mu, lambda, young, nu by Voigt average (fft_fftw_slab.cpp:483-491)."""
    mu = C44 - (2.0 * C44 + C12 - C11) / 5.0
    ll = C12 - (2.0 * C44 + C12 - C11) / 5.0
    young = mu * (3 * ll + 2 * mu) / (ll + mu)
    xnu = young / 2.0 / mu - 1.0
    return mu, ll, young, xnu


def material_constants(mu_in: float, young_in: float):
    """C44, C12, C11 from the deck's mu/young (material.cpp:148-156)."""
    C44 = mu_in
    nu = young_in / 2.0 / mu_in - 1.0
    C12 = 2.0 * nu * C44 / (1.0 - 2.0 * nu)
    C11 = 2.0 * C44 + C12
    return C44, C12, C11


def frequencies(nx: int, ny: int, nz: int, four: np.ndarray):
    """Per-site wavevector fx, fy, fz (fft_fftw_slab.cpp:280-337).

    Index i >= n/2 maps to (i - n)/n, else i/n; the vector is
    k = kx*four[0] + ky*four[1] + kz*four[2].
    """
    def axis(n):
        i = np.arange(n, dtype=np.float64)
        return np.where(i >= n // 2, (i - n) / n, i / n)
    kx, ky, kz = np.meshgrid(axis(nx), axis(ny), axis(nz), indexing="ij")
    four = np.asarray(four, dtype=np.float64)
    fx = kx * four[0, 0] + ky * four[1, 0] + kz * four[2, 0]
    fy = kx * four[0, 1] + ky * four[1, 1] + kz * four[2, 1]
    fz = kx * four[0, 2] + ky * four[1, 2] + kz * four[2, 2]
    return fx, fy, fz


def slip_eigenstrain(xn: np.ndarray, xb: np.ndarray, dslip: float) -> np.ndarray:
    """eps^a_ij = xb_a,i * xn_a,j / dslip (fft_fftw_slab.cpp:559-566)."""
    return np.einsum("ai,aj->aij", xb, xn) / dslip


def bmatrix(nx, ny, nz, four, xn, xb, C44, C12, C11, dslip, chunk=8):
    """BB[a, b, x, y, z] (fft_fftw_slab.cpp:466-638).

    A_mnuv(k) = C_mnuv - C_kluv C_ijmn G_ki k_j k_l with
    G_ki = (2 delta_ik / k^2 - k_i k_k / ((1 - nu) k^4)) / (2 C44), and
    B_ab = A_mnuv eps^a_mn eps^b_uv / mu; A = 0 at k = 0 (first point).
    """
    C = stiffness(C44, C12)
    mu, ll, young, xnu = voigt_constants(C44, C12, C11)
    eps = slip_eigenstrain(np.asarray(xn, float), np.asarray(xb, float), dslip)
    S = eps.shape[0]
    fx, fy, fz = frequencies(nx, ny, nz, four)
    BB = np.empty((S, S, nx, ny, nz))
    for x0 in range(0, nx, chunk):
        k = np.stack([fx[x0:x0 + chunk], fy[x0:x0 + chunk], fz[x0:x0 + chunk]], axis=-1)
        k2 = np.einsum("...i,...i->...", k, k)
        nz_mask = k2 > 0
        k2s = np.where(nz_mask, k2, 1.0)
        eye = np.eye(3)
        G = (2.0 * eye / k2s[..., None, None]
             - (1.0 / (1.0 - xnu)) * np.einsum("...i,...k->...ki", k, k) / (k2s ** 2)[..., None, None]
             ) / (2.0 * C44)
        # Ck = C_ijmn k_j  -> [.., i, m, n];  Cl = C_kluv k_l -> [.., k, u, v]
        Ck = np.einsum("ijmn,...j->...imn", C, k)
        Cl = np.einsum("kluv,...l->...kuv", C, k)
        A = C - np.einsum("...kuv,...ki,...imn->...mnuv", Cl, G, Ck)
        A = np.where(nz_mask[..., None, None, None, None], A, 0.0)
        Ae = np.einsum("...mnuv,buv->...bmn", A, eps)
        B = np.einsum("...bmn,amn->ab...", Ae, eps) / mu
        BB[:, :, x0:x0 + chunk] = B
    return BB


# ---------------------------------------------------------------- stress
def rotate_stress(sigma, prim, invprim, norvol):
    """sigma_rot (fft_fftw_slab.cpp:242-274): rotated when |det prim| ~ 1."""
    sigma = np.asarray(sigma, float)
    if 0.99 < abs(norvol) < 1.01:
        return np.asarray(prim) @ sigma @ np.asarray(invprim)
    return sigma.copy()


def resolved_shear(sigma_rot, xn, xb, dslip):
    """tau_a = sum_ij sigma_rot_ij xn_a,j xb_a,i / dslip (fft_fftw_slab.cpp:737-769)."""
    return np.einsum("ij,aj,ai->a", np.asarray(sigma_rot), np.asarray(xn), np.asarray(xb)) / dslip


def non_schmid_projections(xb, angle_to_110, w1, w2, w3):
    """S_tot[a, i, j] of resolSS_non_Schmid (fft_fftw_slab.cpp:774-840): the
    maximum resolved shear stress plane n at angle_to_110 + 120 a degrees
    (rotation about y), the plane n' 60 degrees from it, and
    S_tot_ij = n_j b_i + w1 n'_j b_i + w2 n_j (n x b)_i + w3 n'_j (n' x b)_i.
    The reference's tables hold three systems."""
    xb = np.asarray(xb, float)
    S = xb.shape[0]
    if S > 3:
        raise ValueError("resolSS_non_Schmid holds at most three systems")
    out = np.zeros((S, 3, 3))
    for a in range(S):
        th = 120.0 * a
        n = np.array([-math.sin((th + angle_to_110) * PI / 180.0), 0.0, math.cos((th + angle_to_110) * PI / 180.0)])
        npl = np.array([-math.sin((th + angle_to_110 + 60) * PI / 180.0), 0.0,
                        math.cos((th + angle_to_110 + 60) * PI / 180.0)])
        b = xb[a]
        nb, npb = np.cross(n, b), np.cross(npl, b)
        out[a] = (np.outer(b, n) + w1 * np.outer(b, npl) + w2 * np.outer(nb, n) + w3 * np.outer(npb, npl))
    return out


def resolved_shear_non_schmid(sigma_rot, xb, dslip, angle_to_110, w1, w2, w3):
    """tau_a = sum_ij sigma_rot_ij S_tot[a, i, j] / dslip (fft_fftw_slab.cpp:812-827)."""
    P = non_schmid_projections(xb, angle_to_110, w1, w2, w3)
    return np.einsum("ij,aij->a", np.asarray(sigma_rot), P) / dslip


def usfe_angle_tau(sigma_rot, mu, fit, angle_to_110):
    """Core model 6 amplitude An (J/m^2) of core_energy_USFE_angle_tau
    (fft_fftw_slab.cpp:1517-1528): the fitted USFE in mJ/m^2 at the MRSSP angle
    and the shear stress sigma_rot[2][1] mu (in GPa through the 1e-9), times 1e-3.
    fit = (a_slope, a_b, b_b, c_slope, c_b)."""
    a_slope, a_b, b_b, c_slope, c_b = (float(v) for v in fit)
    t = float(np.asarray(sigma_rot)[2, 1]) * mu * 1.0E-9
    gsfe = (a_slope * t + a_b) * math.sin(b_b * angle_to_110 * PI / 180.0) + (c_slope * t + c_b)
    return gsfe * 1.0E-3


def core_profile(xr, xb, n_planes):
    """project_core_energy (fft_fftw_slab.cpp:1550-1624) on Re xi [S, nx, ny, nz]:
    delta_p = Re xi_p for one or two systems, else the projection
    sum_c (xi_3p b_0c + xi_3p+1 b_1c + xi_3p+2 b_2c) b_1c (the reference reads
    systems 3p..3p+2 with the Burgers vectors of systems 0..2; planes with
    3p + 2 >= S read past its array and are not defined).  ddelta_p is the
    forward difference along x on the line j = ny/2, k = nz/2 (dx = 1, zero at
    the last x of a single-rank run).  Returns delta [NP, nx, ny, nz], ddelta [NP, nx]."""
    xr = np.asarray(xr, float)
    xb = np.asarray(xb, float)
    S, nx, ny, nz = xr.shape
    delta = np.zeros((n_planes, nx, ny, nz))
    for p in range(n_planes):
        if S <= 2:
            delta[p] = xr[p]
        else:
            x0, x1, x2 = xr[3 * p], xr[3 * p + 1], xr[3 * p + 2]
            delta[p] = ((x0 * xb[0, 0] + x1 * xb[1, 0] + x2 * xb[2, 0]) * xb[1, 0]
                        + (x0 * xb[0, 1] + x1 * xb[1, 1] + x2 * xb[2, 1]) * xb[1, 1]
                        + (x0 * xb[0, 2] + x1 * xb[1, 2] + x2 * xb[2, 2]) * xb[1, 2])
    line = delta[:, :, ny // 2, nz // 2]
    ddelta = np.zeros((n_planes, nx))
    ddelta[:, :-1] = (line[:, 1:] - line[:, :-1]) / 1.0
    return delta, ddelta


# ---------------------------------------------------------------- strain / stress diagnostics
def strain_stress(nx, ny, nz, four, xn, xb, dslip, C44, C12, C11, sigma_rot, xi):
    """The reference's strain and stress diagnostics of state xi, computed as
    DiagStress does (diag_stress.cpp:43-62) when data_fftw holds the forward
    transform of xi: Fmatrix (fft_fftw_slab.cpp:644-732), strain (:3370-3469)
    with stressfree_strain (:3252-3326), total_average_strain (:3331-3365) and
    stress (:3474-3553).

    F[s,i,j](k) = sum_klmn C_klmn G_jk eps^s_mn k_i k_l with
    G = (2 I / k^2 - k k^T / ((1 - nu) k^4)) / (2 mu) (Voigt mu, nu), F(0) = 0;
    strain_ij = IFFT(sum_s F[s,i,j] FFT(xi_s)) / N, plus avepst_ij on the real
    part; eps = (strain + strain^T) / 2; sigma_ij = C_ijml (Re strain_ml -
    eps0_ml - avepsts_ml) + sigma_rot_ij mu with eps0 = sum_s eps^s Re xi_s;
    avepsts = S : sigma_rot mu (S the isotropic compliance of material.cpp:
    154-156, here from the Voigt young and nu, identical for isotropic C),
    avepst = avepsts + <eps0>.

    Returns eps [3,3,nx,ny,nz] complex (data_eps), sigma [3,3,nx,ny,nz] real,
    ave_eps [3,3], ave_sigma [3,3], avepst [3,3].
    """
    xi = np.asarray(xi)
    C = stiffness(C44, C12)
    mu, ll, young, xnu = voigt_constants(C44, C12, C11)
    S11, S12 = 1.0 / young, -xnu / young
    S44 = 2.0 * (S11 - S12)
    d = np.eye(3)
    Sc = (S44 / 4.0 * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
          + S12 * np.einsum("ij,kl->ijkl", d, d))
    eps = slip_eigenstrain(np.asarray(xn, float), np.asarray(xb, float), dslip)
    sig = np.einsum("klmn,smn->skl", C, eps)
    fx, fy, fz = frequencies(nx, ny, nz, four)
    k = np.stack([fx, fy, fz], axis=0)                                  # [3, ...]
    k2 = np.einsum("i...,i...->...", k, k)
    nzm = k2 > 0
    k2s = np.where(nzm, k2, 1.0)
    G = (2.0 * d[:, :, None, None, None] / k2s
         - (1.0 / (1.0 - xnu)) * np.einsum("j...,k...->jk...", k, k) / k2s ** 2) / (2.0 * mu)
    X = np.fft.fftn(xi, axes=(1, 2, 3))
    Y = np.einsum("skl,l...,s...->k...", sig, k, X)                     # sum_s (sigma^s k) X_s
    GU = np.einsum("jk...,k...->j...", G, Y)
    Fx = np.einsum("i...,j...->ij...", k, GU) * nzm
    strain = np.fft.ifftn(Fx, axes=(2, 3, 4))
    N = nx * ny * nz
    ave_epsd = np.einsum("sij,s->ij", eps, xi.real.reshape(len(eps), -1).sum(axis=1)) / N
    avepsts = np.einsum("ijkl,kl->ij", Sc, np.asarray(sigma_rot, float)) * mu
    avepst = avepsts + ave_epsd
    strain = strain + avepst[:, :, None, None, None]
    eps_out = 0.5 * (strain + strain.transpose(1, 0, 2, 3, 4))
    ave_eps = eps_out.real.reshape(3, 3, -1).mean(axis=2)
    eps0 = np.einsum("sij,s...->ij...", eps, xi.real)
    sigma = (np.einsum("ijml,ml...->ij...", C, strain.real - eps0 - avepsts[:, :, None, None, None])
             + (np.asarray(sigma_rot, float) * mu)[:, :, None, None, None])
    ave_sigma = sigma.reshape(3, 3, -1).mean(axis=2)
    return eps_out, sigma, ave_eps, ave_sigma, avepst


# ---------------------------------------------------------------- core energy
@dataclass
class CoreModel:
    """GSFE core model; constants in the reference's SI units (J/m^2, Pa, m).

    flag: 1 perfect (fft_fftw_slab.cpp:1130-1191), 2 extended (:1243-1354),
    3 sine (:1360-1418), 4 pyrII (:1429-1493), 5 BCC perfect with the
    edge/screw angle of FFTW_Slab::gradient (:1070-1125, :869-1065; needs
    geom = (four, xn, xb)), 6 USFE(angle, tau)
    (:1500-1545, An = usfe_angle_tau(...) of the stress state), 7 mpea (:1196-1235), and
    103 = sine with a per-site multiplier on isf and usf (random-alloy GSFE;
    no reference counterpart, reduces to flag 3 when the multiplier is 1).
    """
    flag: int
    mu: float              # Material::mu after Bmatrix (Voigt)
    dslip: float
    b: float
    isf: float = 0.0
    usf: float = 0.0
    An: float = 0.0
    c: tuple = (0.0,) * 7          # c0 c1 c2 c3 c4 a1 a3
    aa: tuple = (0.0,) * 5         # aa0..aa4
    bb: tuple = (0.0,) * 4         # bb1..bb4
    site: np.ndarray | None = field(default=None, repr=False)  # A_mpea or multiplier, [S, nx, ny, nz]
    geom: tuple | None = field(default=None, repr=False)       # (four, xn, xb) for flag 5

    def scale(self):
        return self.mu * self.dslip * self.b

    def derivative(self, xr: np.ndarray) -> np.ndarray:
        """dE_core[a, r] from Re xi [S, nx, ny, nz]."""
        s = self.scale()
        f = self.flag
        if f in (1, 6):
            An = self.An / s
            return An * PI * np.sin(2.0 * PI * xr)
        if f == 3:
            isf = self.isf / s
            Cn = (self.usf - isf / 2.0) / s
            return isf * PI * np.sin(2 * PI * xr) + Cn * 2 * PI * np.sin(4 * PI * xr)
        if f == 103:
            m = self.site
            isf = self.isf * m / s
            Cn = (self.usf * m - isf / 2.0) / s
            return isf * PI * np.sin(2 * PI * xr) + Cn * 2 * PI * np.sin(4 * PI * xr)
        if f == 7:
            return self.site / s * PI * np.sin(2.0 * PI * xr)
        if f == 5:
            return self.usf / s * self._bcc_cof(xr) * PI * np.sin(2.0 * PI * xr)
        if f == 4:
            aa = np.asarray(self.aa, dtype=float) / s
            bb = np.asarray(self.bb, dtype=float) / s
            out = np.zeros_like(xr)
            S = xr.shape[0]
            last = xr.reshape(S, -1)[:, -1]
            v = sum((2.0 * PI * (n + 1)) * (bb[n] * np.cos(2.0 * PI * (n + 1) * last)
                                             - aa[n + 1] * np.sin(2.0 * PI * (n + 1) * last))
                    for n in range(4))
            out.reshape(S, -1)[:, -1] = v
            return out
        if f == 2:
            return self._extended_derivative(xr)
        raise ValueError("core model %d not restated" % f)

    def _bcc_cof(self, xr):
        """cof(theta) of core_energy_bcc_perfect (fft_fftw_slab.cpp:1108-1117) with
        theta from FFTW_Slab::gradient (:869-1065): periodic central
        differences, the in-place transform by `four` (later rows use the
        already transformed components), t = grad x n, theta = acos(t.b/|t|),
        pi - theta where (b x t).n < 0, theta = -1 where |t| <= 0.1."""
        four, xn, xb = (np.asarray(v, float) for v in self.geom)
        g = [(np.roll(xr, -1, axis=ax) - np.roll(xr, 1, axis=ax)) / 2 for ax in (1, 2, 3)]
        gx, gy, gz = g
        gx = gx * four[0, 0] + gy * four[1, 0] + gz * four[2, 0]
        gy = gx * four[0, 1] + gy * four[1, 1] + gz * four[2, 1]
        gz = gx * four[0, 2] + gy * four[1, 2] + gz * four[2, 2]
        n = xn[:, :, None, None, None]
        b = xb[:, :, None, None, None]
        t0 = gy * n[:, 2] - gz * n[:, 1]
        t1 = gz * n[:, 0] - gx * n[:, 2]
        t2 = gx * n[:, 1] - gy * n[:, 0]
        mag = np.sqrt(t0 * t0 + t1 * t1 + t2 * t2)
        small = mag <= 0.1
        m = np.where(small, 1.0, mag)
        t0, t1, t2 = t0 / m, t1 / m, t2 / m
        th = np.arccos(np.clip(t0 * b[:, 0] + t1 * b[:, 1] + t2 * b[:, 2], -1.0, 1.0))
        dirv = (b[:, 1] * t2 - b[:, 2] * t1) * n[:, 0] + (b[:, 2] * t0 - b[:, 0] * t2) * n[:, 1] + \
               (b[:, 0] * t1 - b[:, 1] * t0) * n[:, 2]
        th = np.where(dirv < 0.0, np.arccos(-1.0) - th, th)
        th = np.where(small, -1.0, th)
        return np.where(th < 0.0, 1.0, np.where(th < 1.23, 1.1603 * th * th - 2.0431 * th + 1,
                                                   0.5473 * th * th - 2.0035 * th + 1.8923))

    def _extended_derivative(self, xr):
        c0, c1, c2, c3, c4, a1, a3 = (v / self.mu for v in self.c)
        db = self.dslip * self.b
        S = xr.shape[0]
        out = np.empty_like(xr)
        tp = 2.0 * PI
        fp = 4.0 * PI
        for p in range(S // 3):
            x1, x2, x3 = xr[3 * p], xr[3 * p + 1], xr[3 * p + 2]
            sin, cos = np.sin, np.cos
            d1 = (tp / db) * (
                c1 * (sin(tp * (x2 - x1)) + sin(tp * (x3 - x1)))
                + c2 * (2.0 * sin(tp * (x2 + x3 - 2.0 * x1)) + sin(tp * (2.0 * x2 - x3 - x1))
                        + sin(tp * (2.0 * x3 - x1 - x2)))
                + (2.0 * c3) * (sin(fp * (x2 - x1)) + sin(fp * (x3 - x1)))
                + c4 * (3.0 * sin(tp * (x2 + 2.0 * x3 - 3.0 * x1)) + 3.0 * sin(tp * (2.0 * x2 + x3 - 3.0 * x1))
                        + 2.0 * sin(tp * (3.0 * x2 - x3 - 2.0 * x1)) + sin(tp * (3.0 * x2 - 2.0 * x3 - x1))
                        + sin(tp * (3.0 * x3 - x1 - 2.0 * x2)) + 2.0 * sin(tp * (3.0 * x3 - 2.0 * x1 - x2)))
                + a1 * (cos(tp * (x1 - x2)) - cos(tp * (x3 - x1)))
                + (2.0 * a3) * (cos(fp * (x1 - x2)) - cos(fp * (x3 - x1))))
            d2 = (tp / db) * (
                c1 * (sin(tp * (x1 - x2)) + sin(tp * (x3 - x2)))
                + c2 * (sin(tp * (2.0 * x1 - x2 - x3)) + 2.0 * sin(tp * (x3 + x1 - 2.0 * x2))
                        + sin(tp * (2.0 * x3 - x1 - x2)))
                + (2.0 * c3) * (sin(fp * (x1 - x2)) + sin(fp * (x3 - x2)))
                + c4 * (sin(tp * (3.0 * x1 - x2 - 2.0 * x3)) + 2.0 * sin(tp * (3.0 * x1 - 2.0 * x2 - x3))
                        + 3.0 * sin(tp * (x3 + 2.0 * x1 - 3.0 * x2)) + 3.0 * sin(tp * (2.0 * x3 + x1 - 3.0 * x2))
                        + 2.0 * sin(tp * (3.0 * x3 - x1 - 2.0 * x2)) + sin(tp * (3.0 * x3 - 2.0 * x1 - x2)))
                + a1 * (cos(tp * (x2 - x3)) - cos(tp * (x1 - x2)))
                + (2.0 * a3) * (cos(fp * (x2 - x3)) - cos(fp * (x1 - x2))))
            d3 = (tp / db) * (
                c1 * (sin(tp * (x2 - x3)) + sin(tp * (x1 - x3)))
                + c2 * (sin(tp * (2.0 * x1 - x2 - x3)) + sin(tp * (2.0 * x2 - x3 - x1))
                        + 2.0 * sin(tp * (x1 + x2 - 2.0 * x3)))
                + (2.0 * c3) * (sin(fp * (x2 - x3)) + sin(fp * (x1 - x3)))
                + c4 * (2.0 * sin(tp * (3.0 * x1 - x2 - 2.0 * x3)) + sin(tp * (3.0 * x1 - 2.0 * x2 - x3))
                        + sin(tp * (3.0 * x2 - x3 - 2.0 * x1)) + 2.0 * sin(tp * (3.0 * x2 - 2.0 * x3 - x1))
                        + 3.0 * sin(tp * (x1 + 2.0 * x2 - 3.0 * x3)) + 3.0 * sin(tp * (2.0 * x1 + x2 - 3.0 * x3)))
                + a1 * (cos(tp * (x3 - x1)) - cos(tp * (x2 - x3)))
                + (2.0 * a3) * (cos(fp * (x3 - x1)) - cos(fp * (x2 - x3))))
            out[3 * p], out[3 * p + 1], out[3 * p + 2] = d1, d2, d3
        return out

    def energy_density(self, xr: np.ndarray) -> np.ndarray:
        """f(xi) per site-slip, the integral of derivative() (no reference
        counterpart is ever reduced: E_core is accumulated but not output)."""
        s = self.scale()
        f = self.flag
        if f in (1, 6):
            return self.An / s * np.sin(PI * xr) ** 2
        if f == 3:
            isf = self.isf / s
            Cn = (self.usf - isf / 2.0) / s
            return isf * np.sin(PI * xr) ** 2 + Cn * np.sin(2 * PI * xr) ** 2
        if f == 103:
            m = self.site
            isf = self.isf * m / s
            Cn = (self.usf * m - isf / 2.0) / s
            return isf * np.sin(PI * xr) ** 2 + Cn * np.sin(2 * PI * xr) ** 2
        if f == 7:
            return self.site / s * np.sin(PI * xr) ** 2
        if f == 5:   # usf' cof(theta) sin^2(pi xi), as core_energy_bcc_perfect accumulates it (:1119)
            return self.usf / s * self._bcc_cof(xr) * np.sin(PI * xr) ** 2
        if f == 2:   # fcore of each plane of three systems (:1320), on the plane's first system
            c0, c1, c2, c3, c4, a1, a3 = (v / self.mu for v in self.c)
            db = self.dslip * self.b
            out = np.zeros_like(xr)
            cos, sin, tp, fp = np.cos, np.sin, 2.0 * PI, 4.0 * PI
            for p in range(xr.shape[0] // 3):
                x1, x2, x3 = xr[3 * p], xr[3 * p + 1], xr[3 * p + 2]
                out[3 * p] = (c0 + c1 * (cos(tp * (x1 - x2)) + cos(tp * (x2 - x3)) + cos(tp * (x3 - x1)))
                              + c2 * (cos(tp * (2.0 * x1 - x2 - x3)) + cos(tp * (2.0 * x2 - x3 - x1))
                                      + cos(tp * (2.0 * x3 - x1 - x2)))
                              + c3 * (cos(fp * (x1 - x2)) + cos(fp * (x2 - x3)) + cos(fp * (x3 - x1)))
                              + c4 * (cos(tp * (3.0 * x1 - x2 - 2.0 * x3)) + cos(tp * (3.0 * x1 - 2.0 * x2 - x3))
                                      + cos(tp * (3.0 * x2 - x3 - 2.0 * x1)) + cos(tp * (3.0 * x2 - 2.0 * x3 - x1))
                                      + cos(tp * (3.0 * x3 - x1 - 2.0 * x2)) + cos(tp * (3.0 * x3 - 2.0 * x1 - x2)))
                              + a1 * (sin(tp * (x1 - x2)) + sin(tp * (x2 - x3)) + sin(tp * (x3 - x1)))
                              + a3 * (sin(fp * (x1 - x2)) + sin(fp * (x2 - x3)) + sin(fp * (x3 - x1)))) / db
            return out
        raise ValueError("energy of core model %d not restated" % f)


# ---------------------------------------------------------------- the step
@dataclass
class Instance:
    nx: int
    ny: int
    nz: int
    BB: np.ndarray          # [S, S, nx, ny, nz]
    tau: np.ndarray         # [S]
    cd_dt: float            # App::CD * App::timestep
    core: CoreModel
    xo: np.ndarray | None = None   # [S, nx, ny, nz], 1 = frozen

    @property
    def S(self):
        return self.BB.shape[0]

    @property
    def N(self):
        return self.nx * self.ny * self.nz


def gl_step(inst: Instance, xi: np.ndarray):
    """One GL iteration, SolveGL::iterate body (solve_GL.cpp:92-106).

    xi: complex [S, nx, ny, nz] (real part = the physical order parameter).
    Returns (xi_new, xinorm, xiave).
      core force from the current Re xi         (app.cpp:663-672)
      X = FFT(xi) per slip system, unnormalised  (fft_fftw_slab.cpp:1953-1964)
      R_a = sum_b BB_ab X_b                      (fft_fftw_slab.cpp:1670-1695)
      r = IFFT(R)/N                              (fft_fftw_slab.cpp:2012-2023)
      update where xo == 0                       (fft_fftw_slab.cpp:1746-1790)
    """
    dE = inst.core.derivative(xi.real)
    X = np.fft.fftn(xi, axes=(1, 2, 3))
    R = np.einsum("abxyz,bxyz->axyz", inst.BB, X)
    r = np.fft.ifftn(R, axes=(1, 2, 3))
    cd = inst.cd_dt
    new_re = xi.real - cd * (r.real - inst.tau[:, None, None, None] + dE)
    new_im = xi.imag - cd * r.imag
    if inst.xo is not None:
        upd = inst.xo == 0.0
        new_re = np.where(upd, new_re, xi.real)
        new_im = np.where(upd, new_im, xi.imag)
    xi_new = new_re + 1j * new_im
    xinorm = _xinorm(xi, xi_new, inst.xo)
    xiave = float(new_re.sum())
    return xi_new, xinorm, xiave


def _xinorm(old, new, xo):
    """sqrt(sum |dxi|^2) with the reference's stale 'previous' value on masked
    sites: xirep/xiimp keep the last unmasked site's old value (0 before any),
    in loop order isa, i, j, k (fft_fftw_slab.cpp:1761-1781)."""
    o = old.reshape(-1)
    n = new.reshape(-1)
    if xo is None:
        d = n - o
        return float(math.sqrt(np.sum(d.real ** 2 + d.imag ** 2)))
    upd = (xo.reshape(-1) == 0.0)
    idx = np.where(upd, np.arange(o.size), -1)
    idx = np.maximum.accumulate(idx)
    prev = np.where(idx >= 0, o[np.maximum(idx, 0)], 0.0)
    d = n - prev
    return float(math.sqrt(np.sum(d.real ** 2 + d.imag ** 2)))


def run(inst: Instance, xi0: np.ndarray, steps: int):
    """steps GL iterations at one stress state; returns (xi, xinorms, xiaves)."""
    xi = xi0.astype(np.complex128)
    norms, aves = [], []
    for _ in range(steps):
        xi, xn, xa = gl_step(inst, xi)
        norms.append(xn)
        aves.append(xa)
    return xi, np.array(norms), np.array(aves)


# ---------------------------------------------------------------- energy
def total_energy(inst: Instance, xi: np.ndarray):
    """E = 1/2 <xi, L xi> + sum f(Re xi) - sum tau_a Re xi_a over all sites.

    The reference never reduces an energy (E_core is accumulated and unused,
    fft_fftw_slab.cpp:1399); this is the functional whose gradient is the
    drift of update_order_parameter, data_real/N - tau + dE_core
    (fft_fftw_slab.cpp:1773): L = IFFT B FFT / N is self-adjoint, so
    dE/d Re xi = (L xi)_re - tau + f' and dE/d Im xi = (L xi)_im.
    xi may be complex.  Returns (elastic, core, applied).
    """
    xi = np.asarray(xi)
    X = np.fft.fftn(xi, axes=(1, 2, 3))
    R = np.einsum("abxyz,bxyz->axyz", inst.BB, X)
    Lx = np.fft.ifftn(R, axes=(1, 2, 3))
    el = 0.5 * float(np.real(np.sum(np.conj(xi) * Lx)))
    xr = np.real(xi)
    core = float(np.sum(inst.core.energy_density(xr)))
    app = -float(np.sum(inst.tau[:, None, None, None] * xr))
    return el, core, app


# ---------------------------------------------------------------- conductivity sub-problem
@dataclass
class CondMaterial:
    """Material members the conductivity solver reads (material.h:44-56, the
    preset values of material.cpp:260-275 and siblings, deck keywords
    material.cpp:98-135)."""
    condsigma: float
    alpha_resistivity: float = 0.0
    mfpel: float = 1e-9
    alpha_mfpel: float = 0.0
    dlayer: float = 100e-9
    Rgrain: float = 0.0
    beta_disloc: float = 0.0
    rho_disloc: float = 0.0
    Ngrains: int = 1
    Nlayers: int = 1
    pinterface: float = 0.5


def cond_layers(A: CondMaterial, B: CondMaterial, ny: int, temperature: float):
    """Per-y conductivity of FFTW_Slab::backwardcond (fft_fftw_slab.cpp:2064-2156):
    alternating A/B layers along y (A.Nlayers periods, thicknesses from the
    dlayer volume fraction, integer division of ny by Nlayers as the reference
    does), temperature-corrected layer conductivity sigma_layer and the
    effective sigma_eff with interface, grain-boundary and dislocation
    resistivities.  Returns sigma_eff [ny], sigma_layer [ny]."""
    Vf = B.dlayer / (A.dlayer + B.dlayer)
    Nl = int(A.Nlayers)
    prob = 1.0 - A.pinterface
    per = ny // Nl
    dB = int(round(per * Vf))
    dA = int(round(per * (1.0 - Vf)))
    dT = temperature - 300
    eff = np.zeros(ny)
    lay = np.zeros(ny)
    for j in range(ny):
        M = B if (j % (dA + dB)) >= dA else A
        lay[j] = M.condsigma / (1.0 + M.alpha_resistivity * dT)
        ps = 2 * prob / M.dlayer
        lam = M.mfpel / (1.0 + M.alpha_mfpel * dT)
        ag = (lam * M.Ngrains / M.dlayer) * M.Rgrain / (1 - M.Rgrain)
        rd = M.beta_disloc * M.rho_disloc
        if ps > 0.0:
            ri = (1 / lay[j]) * ((3.0 / 16.0) * lam * ps)
            if M.Ngrains > 1:
                rg = (1 / lay[j]) * (1.0 / (1.0 - 3.0 * ag / 2.0 + 3.0 * ag * ag
                                          - 3.0 * ag ** 3.0 * math.log(1.0 + 1.0 / ag)) - 1.0)
                eff[j] = 1 / ((1 / lay[j]) + (2 * ri + (M.Ngrains - 1) * rg) / (M.Ngrains + 1) + rd)
            else:
                eff[j] = 1 / ((1 / lay[j]) + ri + rd)
        else:
            eff[j] = lay[j]
    return eff, lay


def cond_fields(condxi, four, sigma_eff, El_y, epsilonzero):
    """forwardcond + divcurrent + backwardcond's transforms and current
    (fft_fftw_slab.cpp:1699-1741, 2157-2168): the unnormalised inverse
    transforms a = IFFT(i k_y/k^2 c), b = IFFT(k_y^2/k^2 c), the current
    j = sigma_eff(y) (E_y - a/eps0) (complex, as jcurrent) and <j_y>/E_y."""
    c = np.asarray(condxi, dtype=np.complex128)
    nx, ny, nz = c.shape
    N = nx * ny * nz
    fx, fy, fz = frequencies(nx, ny, nz, four)
    k2 = fx * fx + fy * fy + fz * fz
    ch = np.fft.fftn(c)
    pos = k2 > 0.0
    safe = np.where(pos, k2, 1.0)
    jre = np.where(pos, 0.0 - ch.imag * fy / safe, 0.0)
    jim = np.where(pos, 0.0 + ch.real * fy / safe, 0.0)
    bre = np.where(pos, 0.0 + ch.real * fy * fy / safe, 0.0)
    bim = np.where(pos, 0.0 + ch.imag * fy * fy / safe, 0.0)
    a = np.fft.ifftn(jre + 1j * jim) * N
    b = np.fft.ifftn(bre + 1j * bim) * N
    cs = np.asarray(sigma_eff)[None, :, None]
    j = cs * (El_y - a.real / epsilonzero) + 1j * (-cs * a.imag / epsilonzero)
    return a, b, j, float(np.sum(j.real / N)) / El_y


def cond_step(condxi, four, sigma_eff, sigma_layer, El_y, epsilonzero, timestep):
    """One iteration of the conductivity order parameter as SolveGLCond runs it
    (solve_GL+cond.cpp:96-122): forwardcond, divcurrent (fft_fftw_slab.cpp:1699-1741:
    a = i k_y/k^2 c, b = k_y^2/k^2 c, zero at k = 0), backwardcond's two
    unnormalised inverse transforms and real-space assembly (:2157-2186), and
    update_conduct_order_param (:1795-1834).  Returns the new condxi, condxinorm,
    condxiave and the conductivity <j_y>/El_y of that backwardcond.

    The y-derivative of the layer conductivity is taken on the finished
    profile, (s[j+1] - s[j-1])/2 inside and one-sided at the ends.  The
    reference reads s[j+1] of its stack array before its loop writes it
    (:2108 vs :2176-2181), so its driving term, and condxi from the first
    update on, are undefined; a, b, j and the conductivity of a given state
    are defined and pinned (cond_fields)."""
    c = np.asarray(condxi, dtype=np.complex128)
    nx, ny, nz = c.shape
    N = nx * ny * nz
    jr, br, _, cond = cond_fields(c, four, sigma_eff, El_y, epsilonzero)
    cs = np.asarray(sigma_eff)[None, :, None]
    lay = np.asarray(sigma_layer)
    d = np.empty(ny)
    d[0] = lay[1] - lay[0]
    d[-1] = lay[-1] - lay[-2]
    d[1:-1] = (lay[2:] - lay[:-2]) / 2.0
    d = d[None, :, None]
    cre = (cs / epsilonzero) * br.real + (jr.real / epsilonzero - El_y) * d
    cim = (cs / epsilonzero) * br.imag + (jr.imag / epsilonzero) * d
    new = (c.real - (1e-22 * timestep * (cre / N))) + 1j * (c.imag - (1e-22 * timestep * (cim / N)))
    dn = new - c
    norm = math.sqrt(float(np.sum(dn.real ** 2 + dn.imag ** 2)))
    return new, norm, float(np.sum(new.real)), cond
