"""How well the learned guiding distribution fits the light it should learn.

At a probe point on a surface, the guide network (trained by guided renders
on a lucid_capi.Context) gives a von Mises-Fisher mixture q(w) over incident
directions.  Its training target is the incident radiance: the records
weight each sampled direction by its luminance / pdf, so the loss is
minimised by q(w) proportional to the luminance of L_i(p, w).  The incident
radiance itself is rendered here with the FP64 tracer: the camera is put at
the probe (1 mm off the surface) and the six faces of a cube map are rendered
at 90 degrees; each pixel is one direction bin with its solid angle.

KL(p* || q) over the bins of the hemisphere above the surface then measures
the fit; the same divergence of the cosine density (what BSDF sampling of a
diffuse surface draws) is the baseline a guide has to beat.  Values are in
nats.
"""
from __future__ import annotations

import ctypes

import numpy as np

N_LOBES = 8
KAPPA_MIN, KAPPA_MAX = 0.05, 2000.0


def _cube_faces():
    # (forward, up) of the six faces
    return [((1, 0, 0), (0, 1, 0)), ((-1, 0, 0), (0, 1, 0)), ((0, 1, 0), (0, 0, 1)),
            ((0, -1, 0), (0, 0, -1)), ((0, 0, 1), (0, 1, 0)), ((0, 0, -1), (0, 1, 0))]


def incident_radiance(ctx, p, n, res: int = 32, spp: int = 256, max_depth: int = 8, offset: float = 1e-3):
    """Directions (k, 3), solid angles (k,) and mean RGB radiance (k, 3) of
    the cube-map bins above the surface at p with normal n (FP64 sums of
    `spp` samples per bin, through lucid_cuda_render_f64)."""
    p = np.asarray(p, np.float64)
    n = np.asarray(n, np.float64) / np.linalg.norm(n)
    eye = p + offset * n
    dirs, dws, rads = [], [], []
    t = (np.arange(res) + 0.5) / res * 2.0 - 1.0
    for fwd, up in _cube_faces():
        f, u = np.asarray(fwd, np.float64), np.asarray(up, np.float64)
        r = np.cross(f, u)
        ctx.set_camera(*eye, *f, *u, 90.0)
        img = ctx.render_f64(res, res, res, res, spp, 0, max_depth)[..., :3] / spp
        img = img[::-1]   # render_tile rows are Y-flipped: row 0 of the unflipped image is the top
        # camera ray of pixel (x, y): fwd + right * ndc_x + up * ndc_y, ndc_y from the top
        X, Y = np.meshgrid(t, -t)
        d = f[None, None, :] + X[..., None] * r[None, None, :] + Y[..., None] * u[None, None, :]
        l2 = np.sum(d * d, axis=-1)
        d = d / np.sqrt(l2)[..., None]
        dw = (2.0 / res) ** 2 / l2 ** 1.5   # solid angle of a cube-face pixel
        dirs.append(d.reshape(-1, 3))
        dws.append(dw.reshape(-1))
        rads.append(img.reshape(-1, 3))
    d, dw, rad = np.concatenate(dirs), np.concatenate(dws), np.concatenate(rads)
    keep = d @ n > 0.0
    return d[keep], dw[keep], rad[keep]


def mixture_from_raw(raw):
    """The guide's raw outputs (48) -> (weights (8,), kappas (8,), means (8, 3)),
    as the kernels turn them into a mixture (softmax, softplus + floor and
    cap, normalised means)."""
    raw = np.asarray(raw, np.float64)
    lw = raw[:N_LOBES] - raw[:N_LOBES].max()
    w = np.exp(lw) / np.exp(lw).sum()
    x = raw[N_LOBES:2 * N_LOBES]
    k = np.minimum(np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0)))) + KAPPA_MIN, KAPPA_MAX)
    m = raw[16:16 + 3 * N_LOBES].reshape(N_LOBES, 3)
    ln = np.linalg.norm(m, axis=1)
    mu = np.where(ln[:, None] > 1e-6, m / np.maximum(ln, 1e-30)[:, None], np.array([0.0, 0.0, 1.0]))
    return w, k, mu


def mixture_pdf(w, k, mu, dirs):
    """sum_i w_i kappa_i / (2 pi (1 - e^{-2 kappa_i})) exp(kappa_i (mu_i . d - 1))."""
    norm = k / (2.0 * np.pi * (1.0 - np.exp(-2.0 * k)))
    return (w[None, :] * norm[None, :] * np.exp(k[None, :] * (dirs @ mu.T - 1.0))).sum(axis=1)


def guide_raw(lib, weights, box, p, n, wo):
    """Raw outputs of a guide network with `weights` at point p (world), normal
    n and outgoing direction wo, evaluated by the library's own encoding and
    forward kernels (a standalone lucid_guide_* network on device 0)."""
    lo, hi = (np.asarray(b, np.float64) for b in box)
    ext = hi - lo
    p01 = np.where(ext > 0, (np.asarray(p, np.float64) - lo) / np.where(ext > 0, ext, 1.0), 0.0)
    h = ctypes.c_void_p()
    if lib.lucid_guide_create(0, 1, ctypes.byref(h)) != 0:
        raise RuntimeError("lucid_guide_create failed")
    try:
        w = np.ascontiguousarray(weights, np.float32)
        if lib.lucid_guide_set_params(h, w.ctypes.data, w.size) != 0:
            raise RuntimeError("lucid_guide_set_params failed")
        pa = np.asarray([p01], np.float32)
        na = np.asarray([np.asarray(n) / np.linalg.norm(n)], np.float32)
        woa = np.asarray([np.asarray(wo) / np.linalg.norm(wo)], np.float32)
        n_in = 176
        x = np.zeros((1, n_in), np.float32)
        if lib.lucid_guide_encode(h, pa.ctypes.data, na.ctypes.data, woa.ctypes.data, 1, x.ctypes.data) != 0:
            raise RuntimeError("lucid_guide_encode failed")
        out = np.zeros((1, 48), np.float32)
        if lib.lucid_guide_forward(h, x.ctypes.data, 1, out.ctypes.data) != 0:
            raise RuntimeError("lucid_guide_forward failed")
        return out[0]
    finally:
        lib.lucid_guide_destroy(h)


def kl(p_bins, q_bins):
    """KL(p || q) of two distributions over the same bins (each normalised
    here); bins where p is 0 add nothing."""
    p = np.asarray(p_bins, np.float64)
    q = np.asarray(q_bins, np.float64)
    p = p / p.sum()
    q = q / q.sum()
    m = p > 0
    return float(np.sum(p[m] * np.log(p[m] / np.maximum(q[m], 1e-300))))


def probe(ctx, weights, box, p, n, wo, res=32, spp=256, max_depth=8):
    """Fit of a trained guide (weights, box: ctx.guide_params(), read before
    guiding is turned off for these renders) at one probe: KL of the guide
    and of cosine sampling against the incident-radiance distribution, and
    the share of the guide's mass in the brightest 10 % of the bins (vs the
    target's share there)."""
    dirs, dw, rad = incident_radiance(ctx, p, n, res, spp, max_depth)
    lum = rad @ np.array([0.2126, 0.7152, 0.0722])
    target = np.maximum(lum, 0.0) * dw
    w, k, mu = mixture_from_raw(guide_raw(ctx.lib, weights, box, p, n, wo))
    q = mixture_pdf(w, k, mu, dirs) * dw
    cos = np.maximum(dirs @ (np.asarray(n) / np.linalg.norm(n)), 0.0) * dw
    top = np.argsort(target)[::-1][:max(1, len(target) // 10)]
    return {"kl_guide": kl(target, q), "kl_cosine": kl(target, cos),
            "guide_mass_in_hemisphere": float(q.sum()),
            "top10_target_share": float(target[top].sum() / target.sum()),
            "top10_guide_share": float(q[top].sum() / max(q.sum(), 1e-30)),
            "top10_cosine_share": float(cos[top].sum() / cos.sum())}
