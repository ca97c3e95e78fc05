"""Seeded synthetic particle-image pairs with known displacement.

Follows the reference generator (src/synthetic_data.jl:120-276): particles
are Gaussian images with sigma = d/4 accumulated over a ceil(3 sigma) box
(generate_gaussian_particle!, :176-189), displaced by one forward-Euler step
of the flow evaluated at their launch point (:151-167), rendered into both
frames, then additive Gaussian noise and a clamp at zero (:206-232).
Positions are uniform over the frame extended by a margin so particles enter
and leave at the edges. Random streams are numpy PCG64 seeded per pair.

Flow functions take (x, y) = (column, row) in 1-based pixel coordinates and
return (u, v) = (column, row) displacement.
"""
import math

import numpy as np


def uniform_flow(u, v):
    return lambda x, y: (np.full_like(np.asarray(x, float), u), np.full_like(np.asarray(y, float), v))


def lamb_oseen_flow(center, core_radius, peak_displacement):
    """Lamb-Oseen vortex (form of docs/lit/first_vector_field.jl:29-37) with
    the circulation chosen so the peak tangential displacement is
    `peak_displacement` px. center = (x, y)."""
    cx, cy = center
    rc = float(core_radius)
    # v_theta(r) = G/(2 pi r) (1 - exp(-r^2/rc^2)); its maximum over r
    rs = np.linspace(0.05 * rc, 5 * rc, 20001)
    shape = (1 - np.exp(-rs ** 2 / rc ** 2)) / (2 * math.pi * rs)
    gamma = peak_displacement / shape.max()

    def flow(x, y):
        dx = np.asarray(x, float) - cx
        dy = np.asarray(y, float) - cy
        r2 = dx * dx + dy * dy
        with np.errstate(divide="ignore", invalid="ignore"):
            k = np.where(r2 < 1e-9, gamma / (2 * math.pi * rc ** 2), gamma / (2 * math.pi * r2) * (1 - np.exp(-r2 / rc ** 2)))
        return -k * dy, k * dx

    flow.gamma = gamma
    return flow


def sine_shear_flow(amplitude, wavelength):
    """u = A sin(2 pi y / lambda), v = 0."""
    return lambda x, y: (amplitude * np.sin(2 * math.pi * np.asarray(y, float) / wavelength),
                         np.zeros_like(np.asarray(x, float)))


def poiseuille_flow(nrows, peak):
    """Channel flow along x across the rows: u = peak (1 - ((y - yc)/h)^2)."""
    yc = (nrows + 1) / 2.0
    h = nrows / 2.0
    return lambda x, y: (peak * (1 - ((np.asarray(y, float) - yc) / h) ** 2), np.zeros_like(np.asarray(x, float)))


def _render(shape, rows, cols, inten, sigma):
    nr, nc = shape
    radius = math.ceil(3 * sigma)
    margin = 3 * sigma  # render_particle_image's 3-sigma frame margin
    keep = (cols >= 1 - margin) & (cols <= nc + margin) & (rows >= 1 - margin) & (rows <= nr + margin)
    rows, cols, inten = rows[keep], cols[keep], inten[keep]
    r0 = np.rint(rows).astype(np.int64)
    c0 = np.rint(cols).astype(np.int64)
    idx_parts, val_parts = [], []
    for a in range(-radius, radius + 1):
        for b in range(-radius, radius + 1):
            i = r0 + a
            j = c0 + b
            ok = (i >= 1) & (i <= nr) & (j >= 1) & (j <= nc)
            d2 = (j[ok] - cols[ok]) ** 2 + (i[ok] - rows[ok]) ** 2
            val_parts.append(inten[ok] * np.exp(-d2 / (2 * sigma * sigma)))
            idx_parts.append((i[ok] - 1) + (j[ok] - 1) * nr)
    flat = np.bincount(np.concatenate(idx_parts), weights=np.concatenate(val_parts), minlength=nr * nc)
    return flat.reshape((nr, nc), order="F")


def particle_pair(shape, flow, *, seed, ppp=0.05, sigma=0.65, intensity=(0.5, 1.0), noise=0.01, margin=10.0,
                  dtype=np.float32):
    """Render (imgA, imgB) of `shape` = (rows, cols) for `flow`.

    Returns Fortran-ordered arrays (column-major, like Julia matrices)."""
    nr, nc = shape
    rng = np.random.default_rng(seed)
    area = (nr + 2 * margin) * (nc + 2 * margin)
    n = int(round(ppp * area))
    rows = rng.uniform(1 - margin, nr + margin, n)
    cols = rng.uniform(1 - margin, nc + margin, n)
    inten = rng.uniform(intensity[0], intensity[1], n)
    du, dv = flow(cols, rows)
    A = _render(shape, rows, cols, inten, sigma)
    B = _render(shape, rows + dv, cols + du, inten, sigma)
    if noise > 0:
        A += noise * rng.standard_normal((nr, nc))
        B += noise * rng.standard_normal((nr, nc))
        np.maximum(A, 0.0, out=A)
        np.maximum(B, 0.0, out=B)
    return np.asfortranarray(A, dtype=dtype), np.asfortranarray(B, dtype=dtype)


def to_uint16_12bit(img):
    """12-bit camera counts in UInt16: round(clamp(img, 0, 1) * 4095)."""
    return np.asfortranarray(np.rint(np.clip(img, 0, 1) * 4095).astype(np.uint16))


def from_uint16_12bit(img16):
    return np.asfortranarray(img16.astype(np.float32) / np.float32(4095))


def midpoint_truth(flow, x, y, iterations=8):
    """Flow at the trajectory midpoint of a vector attributed to (x, y)
    (bench/run_benchmarks.jl:199-207): symmetric deformation measures the
    displacement of particles launched at (x, y) - d/2."""
    x = np.asarray(x, float)
    y = np.asarray(y, float)
    x0, y0 = x.copy(), y.copy()
    for _ in range(iterations):
        u, v = flow(x0, y0)
        x0 = x - 0.5 * u
        y0 = y - 0.5 * v
    return flow(x0, y0)


# --- the benchmark configurations ------------------------------------------------

def config0_pair(seed=1000):
    """512 x 512, uniform (2.3, -1.7) px, 0.05 ppp, sigma 0.65, noise 0.01."""
    flow = uniform_flow(2.3, -1.7)
    A, B = particle_pair((512, 512), flow, seed=seed)
    return A, B, flow


def config1_pair(seed=1001):
    """1024 x 1024 Lamb-Oseen vortex, core radius 80 px, 8 px peak, centred."""
    flow = lamb_oseen_flow((512.5, 512.5), 80.0, 8.0)
    A, B = particle_pair((1024, 1024), flow, seed=seed)
    return A, B, flow


def config2_case(seed=1001, noise=0.3, window=16, overlap=8):
    """The differentiation case: the 1024 x 1024 vortex pair and a predictor
    P (gny, gnx, 2) = the true field on the window-centre grid of 16-px
    windows at 50 % overlap (127 x 127 nodes) plus N(0, noise) px.
    Returns A, B, flow, P, grid = (y0, ysp, x0, xsp)."""
    A, B, flow = config1_pair(seed)
    step = window - overlap
    nodes = lambda n: (1 + np.arange((n - window) // step + 1) * step) + (window - 1) / 2.0
    y, x = nodes(A.shape[0]), nodes(A.shape[1])
    X, Y = np.meshgrid(x, y)
    u, v = flow(X, Y)
    rng = np.random.default_rng(seed + 7)
    P = np.stack([u, v], axis=-1) + rng.normal(0.0, noise, (len(y), len(x), 2))
    return A, B, flow, P.astype(np.float32), (float(y[0]), float(step), float(x[0]), float(step))


def config4_frames(n_frames=3, shape=(4096, 4096), seed=1004, peak=6.0, ppp=0.01, noise=0.05, sigma=0.65):
    """The large-frame time series: chained frames of a Poiseuille channel
    flow along x (`peak` px at the centre line) at `ppp` particles per pixel,
    noise sigma `noise`, as 12-bit counts in UInt16 (to_uint16_12bit). Frame
    k + 1 holds frame k's particles moved by the flow once; pair k is
    (frames[k], frames[k + 1]). Returns (frames, flow)."""
    nr, nc = shape
    flow = poiseuille_flow(nr, peak)
    rng = np.random.default_rng(seed)
    margin = 10.0
    left = margin + peak * n_frames  # particles that drift into the frame
    n = int(round(ppp * (nr + 2 * margin) * (nc + margin + left)))
    rows = rng.uniform(1 - margin, nr + margin, n)
    cols = rng.uniform(1 - left, nc + margin, n)
    inten = rng.uniform(0.5, 1.0, n)
    frames = []
    for _ in range(n_frames):
        img = _render(shape, rows, cols, inten, sigma)
        if noise > 0:
            img += noise * rng.standard_normal((nr, nc))
        frames.append(to_uint16_12bit(img))
        du, dv = flow(cols, rows)
        rows, cols = rows + dv, cols + du
    return frames, flow


def config3_pairs(n512=24, n768=24, n2048=16, seed0=1003):
    """The mixed batch: (shape, flow, schedule kind) per pair, drawn from the
    pair seed: sinusoidal shear (A ~ U[1,6], lambda ~ U[128,512]) or a uniform
    translation; schedule [64,32,16] or [48,24]."""
    specs = []
    shapes = [(512, 512)] * n512 + [(768, 1024)] * n768 + [(2048, 2048)] * n2048
    for i, shape in enumerate(shapes):
        rng = np.random.default_rng(seed0 + i)
        if rng.uniform() < 0.5:
            A = rng.uniform(1, 6)
            lam = rng.uniform(128, 512)
            flow = sine_shear_flow(A, lam)
            kind = ("shear", A, lam)
        else:
            u, v = rng.uniform(-4, 4, 2)
            flow = uniform_flow(u, v)
            kind = ("uniform", u, v)
        schedule = "64-32-16" if rng.uniform() < 0.5 else "48-24"
        specs.append(dict(shape=shape, flow=flow, kind=kind, schedule=schedule, seed=seed0 + 1000 + i))
    return specs
