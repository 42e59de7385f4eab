"""Synthetic PFDD workloads (seeded) and the reference decks that describe them.

Each workload is built the way the reference builds one: slip normals and
Burgers vectors as the reference app plugins set them (set_slip), isotropic
elastic constants as Material derives them from mu/young, and a deck in the
reference's own input language so the same case can be run through the
reference sources.  The initial order parameter is generated here (seeded
numpy RNG) and handed to both sides as data.

Workloads (sizes as named; the shapes and value ranges follow the
configurations the headline numbers are quoted on):
  loop64      64^3, 3 systems on one z-normal plane, circular loop r=12 at z=32
              on system 0 plus U(-1e-3, 1e-3) noise, sine GSFE isf 45 / usf 175
              mJ/m^2, sigma_xz = 200 MPa, CD*dt = 0.5
  fcc256      256x256x128, 12 FCC {111}<110> systems, 8 seeded loops with radii
              U[8, 40] cells on random systems, sigma_xz = 300 MPa
  alloy       batched mixed-size instances (32^3..128^3), 3 systems, per-site
              lognormal(0, 0.15) multiplier on isf/usf, sigma U[100, 400] MPa
  edge128     128x128x32, 3 systems, straight edge dislocation + 10-cell
              seeded perturbation (adjoint workload)
  frank_read  2 BCC systems on a 60-degree skewed grid with a pinned segment
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

S3 = math.sqrt(3.0)

# ---------------------------------------------------------------- slip sets
def slip_hcp_basal(oflag: float = 0.0):
    """3 systems, normal z, Burgers at 0 and +-60 degrees (app_3d_hcp_basal.cpp:216-245)."""
    xn = np.array([[0.0, 0.0, 1.0]] * 3)
    t = oflag * math.pi / 2.0
    xb = np.array([[math.cos(t), math.sin(t), 0.0],
                   [math.cos(t + math.pi / 3), math.sin(t + math.pi / 3), 0.0],
                   [math.cos(t - math.pi / 3), math.sin(t - math.pi / 3), 0.0]])
    return xn, xb


def slip_fcc12():
    """12 FCC {111}<110> systems (app_fcc.cpp:211-288)."""
    n = np.array([[1, 1, 1], [-1, 1, 1], [1, -1, 1], [1, 1, -1]], float) / S3
    xn = np.repeat(n, 3, axis=0)
    h = 0.5
    xb = np.array([[-h, h, 0], [0, -h, h], [h, 0, -h],
                   [-h, -h, 0], [h, 0, h], [0, -h, h],
                   [-h, -h, 0], [h, 0, -h], [0, -h, -h],
                   [-h, h, 0], [h, 0, h], [0, -h, -h]], float)
    return xn, xb


def slip_frank_read():
    """2 BCC systems (app_frank_read.cpp:96-120), not rotated by the app."""
    xn = np.array([[0.0, 0.7071, 0.7071], [0.7071, 0.0, 0.7071]])
    xb = np.array([[0.57735, 0.57735, -0.57735]] * 2)
    return xn, xb


def rotate_to_grid(v: np.ndarray, four: np.ndarray) -> np.ndarray:
    """Map vectors onto the reciprocal basis as set_slip does
    (app_fcc.cpp:290-313): v'_i = (v . four[i]) / |four[i]|."""
    nf = np.linalg.norm(four, axis=1)
    return (v @ four.T) / nf


def reciprocal_basis(prim: np.ndarray, sa=1.0, sb=1.0, sc=1.0):
    """four[3][3] and vol from the normalised primitive vectors prim (columns
    are x, y, z; fft.cpp:96-135) scaled by `scale sa sb sc` (app.cpp:383-427)."""
    s = np.array(prim, float) * np.array([sa, sb, sc])[None, :]
    vol = (s[1, 0] * s[2, 1] * s[0, 2] - s[2, 0] * s[1, 1] * s[0, 2] + s[2, 0] * s[0, 1] * s[1, 2]
           - s[0, 0] * s[2, 1] * s[1, 2] + s[0, 0] * s[1, 1] * s[2, 2] - s[1, 0] * s[0, 1] * s[2, 2])
    four = np.empty((3, 3))
    four[0] = [(s[1, 1] * s[2, 2] - s[2, 1] * s[1, 2]), (s[2, 1] * s[0, 2] - s[0, 1] * s[2, 2]),
               (s[0, 1] * s[1, 2] - s[1, 1] * s[0, 2])]
    four[1] = [(s[1, 2] * s[2, 0] - s[2, 2] * s[1, 0]), (s[2, 2] * s[0, 0] - s[0, 2] * s[2, 0]),
               (s[0, 2] * s[1, 0] - s[1, 2] * s[0, 0])]
    four[2] = [(s[1, 0] * s[2, 1] - s[2, 0] * s[1, 1]), (s[2, 0] * s[0, 1] - s[0, 0] * s[2, 1]),
               (s[0, 0] * s[1, 1] - s[1, 0] * s[0, 1])]
    return four / vol, vol


def normalised_prim(x, y, z):
    """prim with unit columns, as `fft_style ... primitive x .. y .. z ..` (fft.cpp:96-135)."""
    p = np.array([x, y, z], float).T
    return p / np.linalg.norm(p, axis=0)[None, :]


# ---------------------------------------------------------------- materials
@dataclass
class Material:
    """Deck-level material: preset name plus keyword overrides (material.cpp:41-156)."""
    preset: str = "Cu"
    mu: float = 48.0e9
    young: float = 128.64e9
    b: float = 3.64e-10 / math.sqrt(2.0)     # Cu preset b = a/sqrt(2), a = 3.64e-10 m
    isf: float = 0.045
    usf: float = 0.175
    An: float = 0.0
    dslip: float = 0.8165
    deck_line: str | None = None   # verbatim `material ...` deck line (preset constants as they are)
    elastic_override: tuple | None = None  # (C44, C12, C11) exactly as a deck produced them
    usfe_fit: tuple | None = None  # a_slope, a_b, b_b, c_slope, c_b of the preset (core model 6)

    def elastic(self):
        if self.elastic_override is not None:
            return tuple(self.elastic_override)
        C44 = self.mu
        nu = self.young / 2.0 / self.mu - 1.0
        C12 = 2.0 * nu * C44 / (1.0 - 2.0 * nu)
        return C44, C12, 2.0 * C44 + C12


# ---------------------------------------------------------------- workloads
@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    app: str                       # reference app_style keyword
    xn: np.ndarray
    xb: np.ndarray
    four: np.ndarray
    prim: np.ndarray
    material: Material
    core_flag: int
    sigma: np.ndarray              # deck units (stress / mu)
    cd_dt: float
    xi0: np.ndarray                # [S, nx, ny, nz] float64
    xo: np.ndarray | None = None
    site: np.ndarray | None = None  # per-site GSFE amplitude/multiplier [S, nx, ny, nz]
    dsigma: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))
    core_extra: dict | None = None  # c (7), aa (5), bb (4) GSFE constants for the extended / pyrII cores
    non_schmid: tuple | None = None  # (angle_to_110 degrees, w1, w2, w3): deck `non_Schmid` (app.cpp:446-459)

    @property
    def S(self):
        return self.xn.shape[0]

    @property
    def N(self):
        return self.nx * self.ny * self.nz

    def deck(self, steps: int, fft_style: str = "fftw_slab", run_T: int = 1) -> str:
        """Reference input deck for this workload (syntax of src/in.fcc-pfdd)."""
        p = self.prim
        m = self.material
        s = self.sigma
        d = self.dsigma
        ortho = np.allclose(p, np.eye(3))
        prim_txt = "" if ortho else (
            " primitive x %r %r %r y %r %r %r z %r %r %r" % tuple(
                float(v) for v in (p[0, 0], p[1, 0], p[2, 0], p[0, 1], p[1, 1], p[2, 1],
                                   p[0, 2], p[1, 2], p[2, 2])))
        lines = [
            "seed 576",
            "app_style %s core_energy %d" % (self.app, self.core_flag),
        ] + ([] if self.non_schmid is None else ["non_Schmid %r %r %r %r" % tuple(
            float(v) for v in self.non_schmid)]) + [
            "fft_style %s pbc 1 1 1 mode 1%s" % (fft_style, prim_txt),
            "dimension 3",
            "lattice sc/6n 1",
            "region box block 0 %d 0 %d 0 %d" % (self.nx, self.ny, self.nz),
            "create_box box",
            "create_sites box",
            m.deck_line or "material preset %s mu %r young %r isf %r usf %r An %r" % (
                m.preset, m.mu, m.young, m.isf, m.usf, m.An),
            "solve_style GL max_iter %d tol 0" % steps,
            "temperature 0",
            "scale 1.0 1.0 1.0",
            "sigma initial %r %r %r %r %r %r delta %r %r %r %r %r %r" % tuple(
                float(v) for v in (s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[0, 2], s[1, 2],
                                   d[0, 0], d[1, 1], d[2, 2], d[0, 1], d[0, 2], d[1, 2])),
            "stats 1e12",
            "run %d" % run_T,
        ]
        return "\n".join(lines) + "\n"


def _sigma(component: str, value: float) -> np.ndarray:
    idx = {"xx": (0, 0), "yy": (1, 1), "zz": (2, 2), "xy": (0, 1), "xz": (0, 2), "yz": (1, 2)}[component]
    s = np.zeros((3, 3))
    s[idx] = value
    s[idx[::-1]] = value
    return s


def _disc(nx, ny, cx, cy, r):
    x = np.arange(nx)[:, None] - cx
    y = np.arange(ny)[None, :] - cy
    return (x * x + y * y) <= r * r


# USFE(MRSSP angle, tau) fits of the Ta and Fe presets (Material::set_constants,
# material.cpp:713-717 and :766-770): a_slope, a_b, b_b, c_slope, c_b
TA_USFE_FIT = (51.59816407, -2.27173784, 0.9979452, -4.16536, 1133.961364)
FE_USFE_FIT = (15.524609942496577, 0.004388435835439675, 0.9934680885709689, -0.9065590784654822,
               944.0633238797747)


def ta_material() -> Material:
    """The Ta preset (material.cpp:697-718): a = 3.3058e-10 m, b = sqrt(3) a / 2."""
    a = 3.3058E-10
    return Material(preset="Ta", mu=70.67E9, young=189.24E9, b=math.sqrt(3.0) * a / 2.0, isf=0.0,
                    usf=950.21E-3, An=0.0, usfe_fit=TA_USFE_FIT)


def bcc_screw_workload(n=16, nz=8, seed=11, sigma_mpa=300.0, angle=10.0, w=(0.3, 0.2, 0.1), core_flag=6,
                       name="bcc_screw"):
    """One BCC system (app 1SBCC: n = (0.7071, 0.7071, 0), b = (-0.57735,
    0.57735, 0.57735) as set_slip writes them, CD = 0.25) in Ta with the
    non-Schmid resolved shear stress and, for core model 6, the USFE(angle,
    tau) amplitude; xi = 1 on a band of the (110) plane through the centre
    plus seeded noise.  sigma_yz and sigma_xz carry the load."""
    m = ta_material()
    prim = np.eye(3)
    four, _ = reciprocal_basis(prim)
    xn = np.array([[0.7071, 0.7071, 0.0]])
    xb = np.array([[-0.57735, 0.57735, 0.57735]])
    rng = np.random.default_rng(seed)
    xi0 = rng.uniform(-1e-3, 1e-3, size=(1, n, n, nz))
    x = np.arange(n)[:, None, None]
    y = np.arange(n)[None, :, None]
    z = np.arange(nz)[None, None, :]
    band = (x + y == n) & (np.abs(z - nz // 2) < max(1, nz // 4))
    xi0[0][np.broadcast_to(band, (n, n, nz))] = 1.0
    sig = _sigma("yz", sigma_mpa * 1e6 / m.mu) + _sigma("xz", 0.5 * sigma_mpa * 1e6 / m.mu)
    return Workload(name, n, n, nz, "1SBCC", xn, xb, four, prim, m, core_flag, sig, 0.25, xi0,
                    non_schmid=(float(angle),) + tuple(float(v) for v in w))


# Electrical members of the Cu and W presets (Material::set_constants,
# material.cpp:269-274 and :726-731) that the conductivity solver reads
CU_COND = dict(condsigma=5.95e7, alpha_resistivity=0.00385, mfpel=39.9e-9, alpha_mfpel=0.00385, Rgrain=0.24,
               beta_disloc=1.3e-25)
W_COND = dict(condsigma=1.855e7, alpha_resistivity=0.0042, mfpel=15.5e-9, alpha_mfpel=0.0042, Rgrain=0.42,
              beta_disloc=7.5e-25)
EPSILON_ZERO = 8.8541878128e-12   # Material::epsilonzero (material.h:53)


@dataclass
class CondCase:
    """A conductivity deck (app cond100B, two layer materials Cu/W alternating
    along y): the Workload of its dislocation field, the two materials as
    pfdd_cond_material values, temperature and E_y."""
    workload: Workload
    A: dict
    B: dict
    temperature: float
    El_y: float

    def deck(self) -> str:
        w = self.workload
        A, B = self.A, self.B
        lines = [
            "seed 576",
            "app_style cond100B core_energy 1",
            "fft_style fftw_slab pbc 1 1 1 mode 1",
            "dimension 3",
            "lattice sc/6n 1",
            "region box block 0 %d 0 %d 0 %d" % (w.nx, w.ny, w.nz),
            "create_box box",
            "create_sites box",
            "material preset Cu El 0.0 %r 0.0 dlayer %r Nlayers %d Ngrains %d pinterface %r rho_disloc %r" % (
                self.El_y, A["dlayer"], A["Nlayers"], A["Ngrains"], A["pinterface"], A["rho_disloc"]),
            "material preset W dlayer %r Ngrains %d rho_disloc %r" % (B["dlayer"], B["Ngrains"], B["rho_disloc"]),
            "solve_style GLCond max_iter 1 tol 0",
            "temperature %r" % self.temperature,
            "scale 1.0 1.0 1.0",
            "sigma initial 0 0 0 0 0 0 delta 0 0 0 0 0 0",
            "stats 1e12",
            "run 1",
        ]
        return "\n".join(lines) + "\n"


def cond_case(nx=8, ny=32, nz=8, n_layers=4, temperature=350.0, El_y=1.0, grains=(3, 2), seed=3):
    """Cu/W multilayer along y on an nx x ny x nz grid (one slip system of app
    cond100B: n = z, b = x, CD = 0.5); the dislocation field is a seeded loop
    that the conductivity sub-problem never reads."""
    m = Material(preset="Cu", mu=48.0e9, young=128.64e9)
    prim = np.eye(3)
    four, _ = reciprocal_basis(prim)
    xn = np.array([[0.0, 0.0, 1.0]])
    xb = np.array([[1.0, 0.0, 0.0]])
    rng = np.random.default_rng(seed)
    xi0 = rng.uniform(-1e-3, 1e-3, size=(1, nx, ny, nz))
    w = Workload("cond", nx, ny, nz, "cond100B", xn, xb, four, prim, m, 1, np.zeros((3, 3)), 0.5, xi0)
    A = dict(CU_COND, dlayer=2e-9, Nlayers=n_layers, Ngrains=grains[0], pinterface=0.4, rho_disloc=1e15)
    B = dict(W_COND, dlayer=1e-9, Nlayers=1, Ngrains=grains[1], pinterface=0.5, rho_disloc=5e14)
    return CondCase(w, A, B, temperature, El_y)


def loop_workload(n=64, radius=12.0, noise=1e-3, seed=576, sigma_mpa=200.0, name="loop64",
                  material: Material | None = None, nz: int | None = None):
    """Circular loop on system 0 in the z = nz/2 plane of an n x n x nz grid
    (nz defaults to n), 3 systems on that plane."""
    m = material or Material()
    nx = ny = n
    nz = n if nz is None else nz
    prim = np.eye(3)
    four, _ = reciprocal_basis(prim)
    xn, xb = slip_hcp_basal()
    xn, xb = rotate_to_grid(xn, four), rotate_to_grid(xb, four)
    rng = np.random.default_rng(seed)
    xi0 = rng.uniform(-noise, noise, size=(3, nx, ny, nz)) if noise > 0 else np.zeros((3, nx, ny, nz))
    disc = _disc(nx, ny, nx / 2.0, ny / 2.0, radius)
    xi0[0, :, :, nz // 2][disc] = 1.0
    return Workload(name, nx, ny, nz, "3d-hcp-basal", xn, xb, four, prim, m, 3,
                    _sigma("xz", sigma_mpa * 1e6 / m.mu), 0.5, xi0)


def fcc_workload(nx=256, ny=256, nz=128, n_loops=8, seed=2024, sigma_mpa=300.0, name="fcc256",
                 material: Material | None = None):
    """12 FCC systems with seeded random loops (radius U[8, 40] cells) placed on
    the z = const plane through a random centre of a random system."""
    m = material or Material()
    prim = np.eye(3)
    four, _ = reciprocal_basis(prim)
    xn, xb = slip_fcc12()
    xn, xb = rotate_to_grid(xn, four), rotate_to_grid(xb, four)
    rng = np.random.default_rng(seed)
    xi0 = np.zeros((12, nx, ny, nz))
    for _ in range(n_loops):
        a = int(rng.integers(0, 12))
        r = float(rng.uniform(8, 40))
        cx, cy, cz = rng.uniform(0, nx), rng.uniform(0, ny), int(rng.integers(0, nz))
        xi0[a, :, :, cz][_disc(nx, ny, cx, cy, r)] = 1.0
    return Workload(name, nx, ny, nz, "fcc", xn, xb, four, prim, m, 3,
                    _sigma("xz", sigma_mpa * 1e6 / m.mu), 0.5, xi0)


def edge_workload(nx=128, ny=128, nz=32, seed=7, perturb=10, sigma_mpa=250.0, isf=0.045, usf=0.175,
                  name="edge128"):
    """Straight edge dislocation (xi_0 = 1 for x < nx/2 on the z = nz/2 plane)
    with a seeded perturbation of the line over `perturb` cells."""
    m = Material(isf=isf, usf=usf)
    prim = np.eye(3)
    four, _ = reciprocal_basis(prim)
    xn, xb = slip_hcp_basal()
    rng = np.random.default_rng(seed)
    xi0 = np.zeros((3, nx, ny, nz))
    shift = np.zeros(ny, dtype=int)
    j0 = int(rng.integers(0, ny - perturb))
    shift[j0:j0 + perturb] = rng.integers(-3, 4, size=perturb)
    for j in range(ny):
        xi0[0, : nx // 2 + shift[j], j, nz // 2] = 1.0
    return Workload(name, nx, ny, nz, "3d-hcp-basal", xn, xb, four, prim, m, 3,
                    _sigma("xz", sigma_mpa * 1e6 / m.mu), 0.5, xi0)


def alloy_instance(n, seed, sigma_mpa, spread=0.15, name="alloy"):
    """One random-alloy instance: n^3, 3 systems, loop r = n/5, per-site
    lognormal(0, spread) multiplier on isf and usf."""
    w = loop_workload(n=n, radius=max(2.0, n / 5.0), noise=1e-3, seed=seed, sigma_mpa=sigma_mpa, name=name)
    rng = np.random.default_rng(seed + 7919)
    w.site = np.exp(spread * rng.standard_normal((w.S, n, n, n)))
    w.core_flag = 103
    return w


def alloy_batch(count=64, sizes=(32, 48, 64, 96, 128), seed=99):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(sizes))
        sig = float(rng.uniform(100, 400))
        out.append(alloy_instance(n, seed=seed * 1000 + i, sigma_mpa=sig, name="alloy%d" % i))
    return out


def frank_read_workload(nx=512, ny=512, nz=64, seg=64, usf=0.300, name="frank_read",
                        sigma_final_mpa=600.0, ramp_steps=20000):
    """2 BCC systems on a 60-degree skewed grid; only the plane j = ny/2 of
    system 0 evolves (xo = 0), every other site is pinned, and a segment of
    `seg` cells along x is seeded with xi = 1 between its pinned ends."""
    m = Material(isf=0.0, usf=usf)
    prim = normalised_prim([1, 0, 0], [0.5, 0.866, 0], [0, 0, 1])
    four, _ = reciprocal_basis(prim)
    xn, xb = slip_frank_read()
    S = 2
    xo = np.ones((S, nx, ny, nz))
    xo[0, :, ny // 2, :] = 0.0
    xi0 = np.zeros((S, nx, ny, nz))
    x0 = nx // 2 - seg // 2
    xi0[0, x0:x0 + seg, ny // 2, nz // 2] = 1.0
    xo[0, x0, ny // 2, nz // 2] = 1.0
    xo[0, x0 + seg - 1, ny // 2, nz // 2] = 1.0
    w = Workload(name, nx, ny, nz, "FrankRead", xn, xb, four, prim, m, 3,
                 np.zeros((3, 3)), 0.35, xi0, xo=xo)
    w.dsigma = _sigma("yz", sigma_final_mpa * 1e6 / m.mu / ramp_steps)
    return w
