"""Seeded synthetic electron bunches (host side, numpy).

The reference draws its initial distributions with GSL
(src/Distribution/Distribution.cpp); no public dataset is involved.  The
bunches used here are Gaussian in position and momentum about a reference
particle at the origin moving along +z, drawn from a counter-based
Philox4x32-10 stream (Salmon et al., SC'11) with one stream per bunch id, and
turned into normals by the Box-Muller transform in FP64.  The same host
arrays feed the CUDA path and the oracle.
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 20261203

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = np.uint32(0x9E3779B9)
_W1 = np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32(counter, key, rounds=10):
    """counter: 4 uint32 arrays; key: 2 uint32 scalars.  Returns 4 uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint32) for c in counter)
    k0, k1 = np.uint32(key[0]), np.uint32(key[1])
    with np.errstate(over="ignore"):
        for r in range(rounds):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
            lo0 = (p0 & _MASK).astype(np.uint32)
            hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
            lo1 = (p1 & _MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            if r != rounds - 1:
                k0 = np.uint32(k0 + _W0)
                k1 = np.uint32(k1 + _W1)
    return c0, c1, c2, c3


def _uniform53(a, b):
    """Two uint32 -> double in (0, 1): 53 random bits, centred in their bin."""
    x = (a.astype(np.uint64) >> np.uint64(5)) * np.uint64(67108864) + (b.astype(np.uint64) >> np.uint64(6))
    return (x.astype(np.float64) + 0.5) / 9007199254740992.0


def standard_normals(n, seed=DEFAULT_SEED, stream=0, block=0):
    """2n standard normals for particles 0..n-1 (two per particle) from
    counter (i, stream, block, 0) and key (seed low, seed high)."""
    i = np.arange(n, dtype=np.uint64)
    key = (np.uint32(seed & 0xFFFFFFFF), np.uint32((seed >> 32) & 0xFFFFFFFF))
    ctr = ((i & _MASK).astype(np.uint32), np.full(n, stream & 0xFFFFFFFF, dtype=np.uint32),
           np.full(n, block, dtype=np.uint32), (i >> np.uint64(32)).astype(np.uint32))
    r0, r1, r2, r3 = philox4x32(ctr, key)
    u1 = _uniform53(r0, r1)
    u2 = _uniform53(r2, r3)
    rad = np.sqrt(-2.0 * np.log(u1))
    ang = 2.0 * np.pi * u2
    return rad * np.cos(ang), rad * np.sin(ang)


def gaussian_bunch(n, sigma=(1e-3, 1e-3, 2e-3), bg_z=10.0, rel_spread=1e-3, bg_perp=1e-3,
                   seed=DEFAULT_SEED, bunch_id=0):
    """Electron bunch about the reference particle.

    Positions: x, y, z ~ N(0, sigma) [m].  Momenta (beta*gamma):
    p_z = bg_z * (1 + rel_spread * N(0,1)), p_x, p_y = bg_perp * N(0,1).
    Returns R, P as (n, 3) float64 arrays (x, y, z per particle, like OPAL's
    Vector_t attributes).
    """
    n = int(n)
    g0, g1 = standard_normals(n, seed, bunch_id, 0)
    g2, g3 = standard_normals(n, seed, bunch_id, 1)
    g4, g5 = standard_normals(n, seed, bunch_id, 2)
    R = np.empty((n, 3), dtype=np.float64)
    P = np.empty((n, 3), dtype=np.float64)
    R[:, 0] = sigma[0] * g0
    R[:, 1] = sigma[1] * g1
    R[:, 2] = sigma[2] * g2
    P[:, 0] = bg_perp * g3
    P[:, 1] = bg_perp * g4
    P[:, 2] = bg_z * (1.0 + rel_spread * g5)
    return R, P


def config_bunch(name, n=None, seed=DEFAULT_SEED, bunch_id=0):
    """The fixed Gaussian recipe of the single-bunch workloads:
    1 nC electrons, sigma = (1, 1, 2) mm, beta*gamma_z = 10 with 1e-3 relative
    spread, transverse beta*gamma sigma 1e-3, dt = 1 ps."""
    sizes = {"c1": (100_000, 32, 100, 0.0), "c2": (1_000_000, 64, 1000, 0.0),
             "c3": (10_000_000, 128, 1000, 0.2)}
    N, mesh, steps, bz = sizes[name]
    if n is not None:
        N = int(n)
    R, P = gaussian_bunch(N, seed=seed, bunch_id=bunch_id)
    return dict(R=R, P=P, N=N, nr=(mesh, mesh, mesh), steps=steps, bz_ext=bz, dT=1e-12,
                Q=-1e-9 / N, ref_pz=10.0, dh=0.02)


def dc_bunch(n, length, sigma_r=1e-3, bg_z=10.0, rel_spread=1e-3, bg_perp=1e-3, seed=DEFAULT_SEED, bunch_id=0):
    """A DC (coasting) beam segment: x, y ~ N(0, sigma_r), z uniform on
    [-length/2, length/2) (53-bit uniforms from the same Philox stream),
    momenta as gaussian_bunch.  The reference's DC-beam runs take their
    distributions from the input deck (Distribution.cpp); this seeded
    stand-in is the shape such a run tracks: a beam whose longitudinal
    extent is about one period of the periodic-z solver.
    Returns R, P (n x 3)."""
    n = int(n)
    g0, g1 = standard_normals(n, seed, bunch_id, 0)
    g3, g4 = standard_normals(n, seed, bunch_id, 1)
    g5, _ = standard_normals(n, seed, bunch_id, 2)
    i = np.arange(n, dtype=np.uint64)
    key = (np.uint32(seed & 0xFFFFFFFF), np.uint32((seed >> 32) & 0xFFFFFFFF))
    ctr = ((i & _MASK).astype(np.uint32), np.full(n, bunch_id & 0xFFFFFFFF, dtype=np.uint32),
           np.full(n, 3, dtype=np.uint32), (i >> np.uint64(32)).astype(np.uint32))
    r0, r1, _, _ = philox4x32(ctr, key)
    u = _uniform53(r0, r1)
    R = np.empty((n, 3), dtype=np.float64)
    P = np.empty((n, 3), dtype=np.float64)
    R[:, 0] = sigma_r * g0
    R[:, 1] = sigma_r * g1
    R[:, 2] = length * (u - 0.5)
    P[:, 0] = bg_perp * g3
    P[:, 1] = bg_perp * g4
    P[:, 2] = bg_z * (1.0 + rel_spread * g5)
    return R, P


def photoinjector_bunch(n, nbins=10, sigma_r=1e-3, z_center=4e-3, sigma_z=0.8e-3, bg_head=1.5, bg_tail=0.5,
                        rel_spread=1e-3, bg_perp=1e-3, seed=DEFAULT_SEED, bunch_id=0):
    """A bunch shortly after emission from a cathode at z = 0, with energy bins.

    The reference's photoinjector runs emit particles from the cathode over
    time and label each with the energy bin of its emission slice
    (src/Distribution/Distribution.cpp, setupEnergyBins / emitParticles); the
    first slice has been accelerated longest.  This seeded stand-in draws
    x, y ~ N(0, sigma_r), z ~ N(z_center, sigma_z) (5 sigma clear of the
    cathode at the defaults), splits the bunch into nbins slices of equal
    count by z (bin 0 at the head) and gives slice b a mean beta*gamma_z
    falling linearly from bg_head (head) to bg_tail (tail), with a
    rel_spread relative spread; transverse beta*gamma ~ N(0, bg_perp).
    Returns R, P (n x 3) and bins (n, int32).
    """
    n = int(n)
    g0, g1 = standard_normals(n, seed, bunch_id, 0)
    g2, g3 = standard_normals(n, seed, bunch_id, 1)
    g4, g5 = standard_normals(n, seed, bunch_id, 2)
    R = np.empty((n, 3), dtype=np.float64)
    P = np.empty((n, 3), dtype=np.float64)
    R[:, 0] = sigma_r * g0
    R[:, 1] = sigma_r * g1
    R[:, 2] = z_center + sigma_z * g2
    order = np.argsort(-R[:, 2], kind="stable")
    bins = np.empty(n, dtype=np.int32)
    bins[order] = (np.arange(n) * nbins // n).astype(np.int32)
    frac = bins / max(nbins - 1, 1)
    bg = bg_head + (bg_tail - bg_head) * frac
    P[:, 0] = bg_perp * g3
    P[:, 1] = bg_perp * g4
    P[:, 2] = bg * (1.0 + rel_spread * g5)
    return R, P, bins


def write_solenoid_map(path, accuracy=30, length=0.3, npts=241, b0=1.0, edge=0.03, width=0.01, jitter=0.0, seed=3):
    """A seeded synthetic on-axis solenoid profile in ASTRA 1D format
    ("AstraMagnetostatic <accuracy>", then "z Bz" lines): a flat top of
    b0 between edge and length - edge with tanh fringes of the given width.
    jitter > 0 moves the sample points off the equidistant grid (the reader
    resamples them by a cubic spline).  Stands in for the field maps of the
    reference's examples, which are not shipped here."""
    z = np.linspace(0.0, length, npts)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dz = length / (npts - 1)
        z[1:-1] += rng.uniform(-jitter, jitter, npts - 2) * dz
    bz = 0.5 * b0 * (np.tanh((z - edge) / width) - np.tanh((z - (length - edge)) / width))
    with open(path, "w") as f:
        f.write(f"AstraMagnetostatic {accuracy}\n")
        for zi, bi in zip(z, bz):
            f.write(f"{zi:.17g} {bi:.17g}\n")
    return z, bz


def write_rfcavity_map(path, accuracy=40, freq_mhz=1300.0, cells=2, npts=301, width=0.01, jitter=0.0, seed=5):
    """A seeded synthetic on-axis E_z profile of a standing-wave cavity in
    ASTRA 1D dynamic format ("AstraDynamic <accuracy>", the frequency in MHz,
    then "z Ez" lines): `cells` pi-mode cells of length c / (2 f),
    E_z = sin(pi z / cell) inside, with tanh fringes of the given width at
    both ends.  Stands in for the reference examples' cavity maps, which are
    not shipped here.  Returns z, Ez."""
    cell = 299792458.0 / (2.0 * freq_mhz * 1e6)
    length = cells * cell
    z = np.linspace(0.0, length, npts)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dz = length / (npts - 1)
        z[1:-1] += rng.uniform(-jitter, jitter, npts - 2) * dz
    env = 0.5 * (np.tanh(z / width) - np.tanh((z - length) / width))
    ez = np.sin(np.pi * z / cell) * env
    with open(path, "w") as f:
        f.write(f"AstraDynamic {accuracy}\n{freq_mhz:.17g}\n")
        for zi, ei in zip(z, ez):
            f.write(f"{zi:.17g} {ei:.17g}\n")
    return z, ez


def write_2d_solenoid_map(path, orientation="XZ", normalize=None, length=0.3, radius=0.04, nz=120, nr=20, b0=1.0,
                          edge=0.04, width=0.012, comment=True):
    """A seeded synthetic solenoid in OPAL's 2DMagnetoStatic format on an
    (r, z) grid (cm): the on-axis field of a tanh-edged coil, Bz(z), with its
    paraxial off-axis expansion Bz = Bz0 - r^2/4 Bz0'', Br = -r/2 Bz0'.
    Stands in for the reference examples' 2D maps, which are not shipped
    here.  orientation "XZ" (r-major "Bz Br" lines) or "ZX" (z-major
    "Br Bz"); normalize None writes no flag, else TRUE / FALSE.  Returns z, r
    [m] and the arrays [r, z]."""
    z = np.linspace(0.0, length, nz + 1)
    r = np.linspace(0.0, radius, nr + 1)
    t1, t2 = np.tanh((z - edge) / width), np.tanh((z - (length - edge)) / width)
    bz0 = 0.5 * b0 * (t1 - t2)
    s1, s2 = 1 - t1 ** 2, 1 - t2 ** 2
    d1 = 0.5 * b0 * (s1 - s2) / width
    d2 = 0.5 * b0 * (-2 * t1 * s1 + 2 * t2 * s2) / width ** 2
    R, _ = np.meshgrid(r, z, indexing="ij")
    BZ = bz0[None, :] - R ** 2 / 4 * d2[None, :]
    BR = -R / 2 * d1[None, :]
    flag = "" if normalize is None else (" TRUE" if normalize else " FALSE")
    with open(path, "w") as f:
        f.write(f"2DMagnetoStatic {orientation}{flag}\n")
        if comment:
            f.write("# synthetic coil: z and r in cm, B in T\n")
        if orientation == "XZ":
            f.write(f"{0.0:.17g} {100 * length:.17g} {nz}\n{0.0:.17g} {100 * radius:.17g} {nr}\n")
            for j in range(nr + 1):
                for i in range(nz + 1):
                    f.write(f"{BZ[j, i]:.17g} {BR[j, i]:.17g}\n")
        else:
            f.write(f"{0.0:.17g} {100 * radius:.17g} {nr}\n{0.0:.17g} {100 * length:.17g} {nz}\n")
            for i in range(nz + 1):
                for j in range(nr + 1):
                    f.write(f"{BR[j, i]:.17g} {BZ[j, i]:.17g}\n")
    return z, r, BZ, BR


def write_2d_rfcavity_map(path, orientation="XZ", normalize=None, freq_mhz=1300.0, cells=2, radius=0.03, nz=160,
                          nr=24, comment=True):
    """A seeded synthetic standing-wave cavity in OPAL's 2DDynamic format on
    an (r, z) grid (cm; E in MV/m, H in A/m): `cells` pi-mode cells of length
    c / (2 f), Ez = sin(pi z / cell) J0-like in r (1 - (k r)^2 / 4),
    Er = -r/2 dEz/dz, H_theta = (omega eps0 r / 2) Ez.  orientation "XZ"
    (r-major "Ez Er |E| Ht") or "ZX" (z-major "Er Ez Ht |E|").  Returns z, r
    [m] and the arrays [r, z]."""
    c = 299792458.0
    cell = c / (2.0 * freq_mhz * 1e6)
    length = cells * cell
    k = 2 * np.pi * freq_mhz * 1e6 / c
    z = np.linspace(0.0, length, nz + 1)
    r = np.linspace(0.0, radius, nr + 1)
    R, Z = np.meshgrid(r, z, indexing="ij")
    ez0 = np.sin(np.pi * Z / cell)
    dez0 = np.pi / cell * np.cos(np.pi * Z / cell)
    EZ = ez0 * (1 - (k * R) ** 2 / 4)
    ER = -R / 2 * dez0
    HT = 2 * np.pi * freq_mhz * 1e6 * 8.854187817e-12 * R / 2 * ez0 * 1e6  # A/m of the MV/m field
    EA = np.sqrt(EZ ** 2 + ER ** 2)
    flag = "" if normalize is None else (" TRUE" if normalize else " FALSE")
    with open(path, "w") as f:
        f.write(f"2DDynamic {orientation}{flag}\n")
        if comment:
            f.write("# synthetic cavity: z and r in cm, E in MV/m, H in A/m\n")
        if orientation == "XZ":
            f.write(f"{0.0:.17g} {100 * length:.17g} {nz}\n{freq_mhz:.17g}\n{0.0:.17g} {100 * radius:.17g} {nr}\n")
            for j in range(nr + 1):
                for i in range(nz + 1):
                    f.write(f"{EZ[j, i]:.17g} {ER[j, i]:.17g} {EA[j, i]:.17g} {HT[j, i]:.17g}\n")
        else:
            f.write(f"{0.0:.17g} {100 * radius:.17g} {nr}\n{freq_mhz:.17g}\n{0.0:.17g} {100 * length:.17g} {nz}\n")
            for i in range(nz + 1):
                for j in range(nr + 1):
                    f.write(f"{ER[j, i]:.17g} {EZ[j, i]:.17g} {HT[j, i]:.17g} {EA[j, i]:.17g}\n")
    return z, r, EZ, ER, HT


def write_3d_rfcavity_map(path, normalize=None, freq_mhz=1300.0, cells=2, half_width=0.02, nx=16, ny=12, nz=80,
                          seed=3, comment=True):
    """A seeded synthetic standing-wave cavity in OPAL's 3DDynamic format on
    an (x, y, z) grid (cm; E in MV/m, H in A/m): the field of
    write_2d_rfcavity_map in Cartesian components (Ez = sin(pi z / cell)
    (1 - (k r)^2 / 4), E_perp = -(x, y)/2 dEz/dz, H = (omega eps0 / 2)
    (-y, x, 0) Ez) plus a seeded perturbation of 1e-3 of each component's
    scale, so that no two grid axes are interchangeable; x in [-w, w] with nx
    intervals, y with ny, z over `cells` cells with nz.  Returns x, y, z [m]
    and the six arrays [component, x, y, z] as written."""
    c = 299792458.0
    cell = c / (2.0 * freq_mhz * 1e6)
    length = cells * cell
    k = 2 * np.pi * freq_mhz * 1e6 / c
    x = np.linspace(-half_width, half_width, nx + 1)
    y = np.linspace(-half_width, half_width, ny + 1)
    z = np.linspace(0.0, length, nz + 1)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    ez0 = np.sin(np.pi * Z / cell)
    dez0 = np.pi / cell * np.cos(np.pi * Z / cell)
    w_eps = 2 * np.pi * freq_mhz * 1e6 * 8.854187817e-12 * 1e6  # A/m per MV/m per m
    F = np.stack([-X / 2 * dez0, -Y / 2 * dez0, ez0 * (1 - k ** 2 * (X ** 2 + Y ** 2) / 4),
                  -w_eps * Y / 2 * ez0, w_eps * X / 2 * ez0, np.zeros_like(Z)])
    rng = np.random.default_rng(seed)
    scale = np.maximum(np.abs(F).reshape(6, -1).max(axis=1), 1e-3 * w_eps * half_width)
    F = F + 1e-3 * scale[:, None, None, None] * rng.standard_normal(F.shape)
    flag = "" if normalize is None else (" TRUE" if normalize else " FALSE")
    with open(path, "w") as f:
        f.write(f"3DDynamic{flag}\n")
        if comment:
            f.write("# synthetic cavity: x, y, z in cm, E in MV/m, H in A/m\n")
        f.write(f"{freq_mhz:.17g}\n")
        f.write(f"{-100 * half_width:.17g} {100 * half_width:.17g} {nx}\n")
        f.write(f"{-100 * half_width:.17g} {100 * half_width:.17g} {ny}\n")
        f.write(f"{0.0:.17g} {100 * length:.17g} {nz}\n")
        rows = F.reshape(6, -1).T
        for r in rows:
            f.write(" ".join(f"{v:.17g}" for v in r) + "\n")
    return x, y, z, F
