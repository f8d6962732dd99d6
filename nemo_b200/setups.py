"""Initial conditions of the benchmark workloads (seeded synthetic data).

Each function returns the conserved state u[V,E,n^3] (float64, Fortran node order i fastest) on the
Gauss-Lobatto nodes of a mesh from nemo_b200.mesh.  Formulas follow the reference setups where one
exists (cited per function); the workload parameters are the benchmark's own.
"""
import numpy as np

from . import mesh as _mesh

LGL4 = np.array([-1.0, -1.0 / np.sqrt(5.0), 1.0 / np.sqrt(5.0), 1.0])


def prim2cons(rho, vx, vy, vz, p, kappa):
    """prim2cons, source/equations/euler/equations_mod.f90:195-208."""
    return np.stack([rho, vx * rho, vy * rho, vz * rho,
                     p / (kappa - 1.0) + 0.5 * rho * (vx ** 2 + vy ** 2 + vz ** 2)])


def density_wave(m, seed=1234, kappa=1.4, noise=1e-3, nodes=LGL4):
    """Smooth periodic case on [0,1]^3: rho = 1 + 0.5 sin(2 pi (x+y+z)) + U(-noise, noise),
    u = v = w = 1, p = 1 (cf. the advected wave of
    source/setups/euler/3d/convergence-test/setup_manufacsol_mod.f90:9-32)."""
    x, y, z = m.node_coords(nodes)
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * (x + y + z)) + rng.uniform(-noise, noise, size=x.shape)
    one = np.ones_like(x)
    return np.ascontiguousarray(prim2cons(rho, one, one, one, one, kappa))


def sedov(m, sigma=0.05, e0=1.0, rho0=1.0, p0=1e-5, kappa=1.4, nodes=LGL4, center=(0.0, 0.0, 0.0)):
    """Sedov-type blast on [-1/2,1/2]^3: ambient rho0, p0 at rest, energy e0 deposited as a normalised
    Gaussian of width sigma (source/setups/euler/3d/sedov/setup_init_mod.f90 and
    setup_config_mod.f90:38-40: E += e0/sqrt((2 pi)^3)/sigma^3 * exp(-r^2/(2 sigma^2)))."""
    x, y, z = m.node_coords(nodes)
    r = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2)
    zero = np.zeros_like(x)
    u = prim2cons(rho0 + zero, zero, zero, zero, p0 + zero, kappa)
    u[4] += e0 / np.sqrt((2 * np.pi) ** 3) / sigma ** 3 * np.exp(-0.5 * (r / sigma) ** 2)
    return np.ascontiguousarray(u)


def gaussian_blob(m, amp, sigma=0.1, kappa=1.4, nodes=LGL4, vel=(0.5, 0.5, 0.5)):
    """Advected Gaussian density blob on [0,1]^3 (source/setups/euler/3d/advecting-gaussian-bell/
    setup_init_mod.f90 form) with amplitude amp: rho = 1 + amp exp(-r^2/(2 sigma^2)), p = 1."""
    x, y, z = m.node_coords(nodes)
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2
    rho = 1.0 + amp * np.exp(-0.5 * r2 / sigma ** 2)
    one = np.ones_like(x)
    return np.ascontiguousarray(prim2cons(rho, vel[0] * one, vel[1] * one, vel[2] * one, one, kappa))


def kelvin_helmholtz(m, seed=7, kappa=1.4, nodes=LGL4, amp=0.01):
    """3D Kelvin-Helmholtz on [-1,1]^3: dense shear layer |y| < 0.25 (rho 2, vx +0.5) between
    rho 1, vx -0.5 (delta u = 1, density ratio 2), p = 2.5, seeded sinusoidal perturbation of vy of
    amplitude amp (after the 2D setup source/setups/euler/2d/kelvin-helmholtz-instability)."""
    x, y, z = m.node_coords(nodes)
    rng = np.random.default_rng(seed)
    kx, kz = rng.integers(1, 4, size=2)
    ph = rng.uniform(0, 2 * np.pi, size=2)
    inside = np.abs(y) < 0.25
    rho = np.where(inside, 2.0, 1.0)
    vx = np.where(inside, 0.5, -0.5)
    vy = amp * np.sin(np.pi * kx * x + ph[0]) * np.sin(np.pi * kz * z + ph[1])
    vz = np.zeros_like(x)
    p = 2.5 * np.ones_like(x)
    return np.ascontiguousarray(prim2cons(rho, vx, vy, vz, p, kappa))


def smooth_random(m, seed=0, kappa=1.4, nodes=LGL4, amp=0.2):
    """Smooth periodic state on [0,1]^3 with distinct, seeded sinusoidal density, velocity components
    and pressure (a parity workload in which no two momentum components coincide)."""
    x, y, z = m.node_coords(nodes)
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, size=(5, 3))
    kk = rng.integers(1, 3, size=(5, 3))

    def wave(i):
        return (np.sin(2 * np.pi * kk[i, 0] * x + ph[i, 0]) * np.cos(2 * np.pi * kk[i, 1] * y + ph[i, 1])
                + np.sin(2 * np.pi * kk[i, 2] * z + ph[i, 2]))

    rho = 1.0 + amp * wave(0)
    vx, vy, vz = 0.5 * wave(1), -0.4 * wave(2), 0.3 * wave(3)
    p = 1.0 + amp * wave(4)
    return np.ascontiguousarray(prim2cons(rho, vx, vy, vz, p, kappa))


def mhd_prim2cons(rho, vx, vy, vz, p, bx, by, bz, psi, kappa, mu0=1.0):
    """Primitive -> conserved GLM-MHD variables (rho, m, E, B, psi) with
    E = p/(kappa-1) + rho v^2/2 + (B^2 + psi^2)/(2 mu0) (source/setups/mhd/3d/orszag-tang/setup_init_mod.f90)."""
    ener = p / (kappa - 1.0) + 0.5 * rho * (vx ** 2 + vy ** 2 + vz ** 2) + 0.5 / mu0 * (bx ** 2 + by ** 2 + bz ** 2) \
        + 0.5 / mu0 * psi ** 2
    return np.stack([rho, rho * vx, rho * vy, rho * vz, ener, bx, by, bz, psi])


def orszag_tang(m, kappa=5.0 / 3.0, eps=0.2, b0=1.0 / np.sqrt(4.0 * np.pi), nodes=LGL4):
    """3D Orszag-Tang-type vortex on the periodic unit box: rho = 25/(36 pi), p = 5/(12 pi),
    v = (-(1 + eps sin 2 pi z) sin 2 pi y, (1 + eps sin 2 pi z) sin 2 pi x, eps sin 2 pi z),
    B = b0 (-sin 2 pi y, sin 4 pi x, 0), psi = 0, mu0 = 1 (the velocity and field pattern of
    source/setups/mhd/3d/orszag-tang/setup_init_mod.f90 with the classic density/pressure/b0)."""
    x, y, z = m.node_coords(nodes)
    tp = 2.0 * np.pi
    rho = np.full_like(x, 25.0 / (36.0 * np.pi))
    p = np.full_like(x, 5.0 / (12.0 * np.pi))
    fz = 1.0 + eps * np.sin(tp * z)
    vx, vy, vz = -fz * np.sin(tp * y), fz * np.sin(tp * x), eps * np.sin(tp * z)
    bx, by, bz = -b0 * np.sin(tp * y), b0 * np.sin(2 * tp * x), np.zeros_like(x)
    return np.ascontiguousarray(mhd_prim2cons(rho, vx, vy, vz, p, bx, by, bz, np.zeros_like(x), kappa))


def divergence_b(m, u, dmat, weights):
    """Discrete div B on the Gauss-Lobatto nodes (D applied along each direction, 2/delta scaling):
    returns (L2 norm over the domain, max |div B|)."""
    E = m.E
    n = dmat.shape[0]
    B = u[5:8].reshape(3, E, n, n, n)  # [c][e][k][j][i]
    div = np.einsum("im,ekjm->ekji", dmat, B[0]) * (2.0 / m.delta[:, 0])[:, None, None, None]
    div += np.einsum("jm,ekmi->ekji", dmat, B[1]) * (2.0 / m.delta[:, 1])[:, None, None, None]
    div += np.einsum("km,emji->ekji", dmat, B[2]) * (2.0 / m.delta[:, 2])[:, None, None, None]
    w3 = np.einsum("k,j,i->kji", weights, weights, weights) / 8.0
    vol = np.prod(m.delta, axis=1)[:, None, None, None]
    l2 = float(np.sqrt(np.sum(w3[None] * vol * div ** 2)))
    return l2, float(np.max(np.abs(div)))
