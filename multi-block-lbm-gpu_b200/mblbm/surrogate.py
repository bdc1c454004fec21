"""Learned warm start of the multi-block solver (no counterpart in the
reference project).

The surrogate (mblbm.UNet, a 4-level convolutional U-Net run by the
library's own tensor-core kernels) maps, on an H x W grid spanning a case's
domain, four input channels (the obstacle's signed distance / D, Re / 100,
the inside-obstacle flag, x / LX) to three outputs (u / U0, v / U0,
100 (rho - 1)).  It is trained on snapshots the solver itself produces
(batched cases of mblbm.batch_case, after a fixed number of coarse steps).
Its prediction initialises every block of a new case: f = feq(rho, u) plus
the Chapman-Enskog non-equilibrium part built from the predicted velocity
gradients, stored post-collision, then the ring slots and u_prev are
re-derived (mb_sync_history).
"""
import numpy as np

from . import (MB_SOLID_SBB, OBST_ELLIPSE, Batch, MultiBlockLBM, UNet, batch_case, updates_per_coarse_step)

H, W = 128, 256
EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)
WK = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def grid_coords(geo, h=H, w=W):
    """Coarse-cell coordinates (X, Y) of the h x w surrogate grid points."""
    c = geo.config
    X = np.linspace(0.0, c.LX - 1.0, w)
    Y = np.linspace(0.0, c.LY - 1.0, h)
    return np.meshgrid(X, Y)


def obstacle_sdf(geo, X, Y):
    """Signed distance to the obstacle in coarse cells (negative inside);
    for an ellipse the scaled radial distance (exact on its minor axis)."""
    c = geo.config
    if c.obstacle == OBST_ELLIPSE:
        dx, dy = X - c.ell_cx, Y - c.ell_cy
        ca, sa = np.cos(c.ell_angle), np.sin(c.ell_angle)
        xr, yr = ca * dx + sa * dy, -sa * dx + ca * dy
        k = np.sqrt((xr / c.ell_a) ** 2 + (yr / c.ell_b) ** 2)
        return (k - 1.0) * min(c.ell_a, c.ell_b)
    return np.sqrt((X - c.CX) ** 2 + (Y - c.CY) ** 2) - c.R


def case_inputs(geo, h=H, w=W):
    """Network input (h, w, 4) float32 and the fluid mask (h, w)."""
    c = geo.config
    X, Y = grid_coords(geo, h, w)
    D = 2.0 * max(c.ell_a, c.ell_b) if c.obstacle == OBST_ELLIPSE else 2.0 * c.R
    sdf = obstacle_sdf(geo, X, Y)
    inside = (sdf < 0).astype(np.float64)
    inp = np.stack([sdf / D, np.full_like(X, c.Re / 100.0), inside, X / (c.LX - 1.0)], axis=-1)
    return inp.astype(np.float32), (1.0 - inside).astype(np.float32)


def coarse_fields(sim, geo):
    """rho, ux, uy on every coarse cell (LY, LX) from the blocks (finer
    levels overwrite coarser ones where they overlap)."""
    c = geo.config
    out = np.full((3, c.LY, c.LX), np.nan)
    L = geo.layout
    for lev in range(L.LEVEL):
        for a in range(L.ASP[lev], L.ASP[lev + 1]):
            A = geo.Areas[a]
            m = A.m
            i0 = int(round((np.ceil(A.base_x - 1e-9) - A.base_x) * m))
            j0 = int(round((np.ceil(A.base_y - 1e-9) - A.base_y) * m))
            X0, Y0 = int(round(A.base_x + i0 / m)), int(round(A.base_y + j0 / m))
            f = sim.macros(a)
            for q, k in enumerate(("rho", "ux", "uy")):
                sub = f[k][j0::m, i0::m]
                out[q, Y0:Y0 + sub.shape[0], X0:X0 + sub.shape[1]] = sub
    return out


def bilinear(field, X, Y):
    """field (ny, nx) at fractional coordinates X, Y (clamped to the grid)."""
    ny, nx = field.shape
    X = np.clip(X, 0, nx - 1)
    Y = np.clip(Y, 0, ny - 1)
    x0 = np.minimum(np.floor(X).astype(int), nx - 2)
    y0 = np.minimum(np.floor(Y).astype(int), ny - 2)
    tx, ty = X - x0, Y - y0
    return ((1 - ty) * ((1 - tx) * field[y0, x0] + tx * field[y0, x0 + 1]) +
            ty * ((1 - tx) * field[y0 + 1, x0] + tx * field[y0 + 1, x0 + 1]))


def case_targets(sim, geo, h=H, w=W):
    """Network target (h, w, 3) float32 from the solver's current fields."""
    rho, ux, uy = coarse_fields(sim, geo)
    U0 = geo.config.U0[0]
    X, Y = grid_coords(geo, h, w)
    t = np.stack([bilinear(ux, X, Y) / U0, bilinear(uy, X, Y) / U0, 100.0 * (bilinear(rho, X, Y) - 1.0)], axis=-1)
    return t.astype(np.float32)


# Reynolds number above which the wake of the workload's obstacles sheds
RE_SHEDDING = 47.0


def wake_kick(cfg, h, w, kick):
    """Transverse velocity (h, w) added to a prediction on the h x w grid of
    warm_start: kick * U0 in a Gaussian of radius R centred 3R behind the
    obstacle at (CX, CY); zero when kick <= 0 or Re < RE_SHEDDING."""
    if kick <= 0.0 or cfg.Re < RE_SHEDDING:
        return np.zeros((h, w))
    gx, gy = (cfg.LX - 1.0) / (w - 1), (cfg.LY - 1.0) / (h - 1)
    yy, xx = np.meshgrid(np.arange(h) * gy, np.arange(w) * gx, indexing="ij")
    r2 = ((xx - (cfg.CX + 3.0 * cfg.R)) ** 2 + (yy - cfg.CY) ** 2) / float(cfg.R) ** 2
    return kick * cfg.U0[0] * np.exp(-r2)


def warm_start(sim, geo, pred, stream=None, kick=0.0):
    """Initialise every block of sim from a prediction (h, w, 3): f = feq +
    (1 - 1/tau) f_neq with f_neq_k = -3 w_k rho tau (e_k e_k - I/3) : grad u
    (Chapman-Enskog, lattice units of the block's level), obstacle cells at
    rest; then ring slots and u_prev follow the new fields.

    kick > 0 (shedding cases, Re >= RE_SHEDDING, only): the surrogate
    predicts the mean wake, which is symmetric, and shedding would have to
    grow out of round-off again; a transverse velocity kick * U0 in a
    Gaussian of radius R centred 3R behind the obstacle breaks the symmetry
    so the wake starts shedding at once."""
    c = geo.config
    U0 = c.U0[0]
    h, w = pred.shape[:2]
    u = pred[..., 0].astype(np.float64) * U0
    v = pred[..., 1].astype(np.float64) * U0
    rho = 1.0 + pred[..., 2].astype(np.float64) / 100.0
    gx, gy = (c.LX - 1.0) / (w - 1), (c.LY - 1.0) / (h - 1)
    v = v + wake_kick(c, h, w, kick)
    dudy, dudx = np.gradient(u, gy, gx)
    dvdy, dvdx = np.gradient(v, gy, gx)
    L = geo.layout
    for a in range(L.number_area):
        A = geo.Areas[a]
        m, tau = A.m, A.tau
        jj, ii = np.meshgrid(np.arange(A.ny), np.arange(A.nx), indexing="ij")
        Xg = (A.base_x + ii / m) / gx
        Yg = (A.base_y + jj / m) / gy
        r = bilinear(rho, Xg, Yg)
        ux, uy = bilinear(u, Xg, Yg), bilinear(v, Xg, Yg)
        sxx, syy = bilinear(dudx, Xg, Yg) / m, bilinear(dvdy, Xg, Yg) / m
        sxy = 0.5 * (bilinear(dudy, Xg, Yg) + bilinear(dvdx, Xg, Yg)) / m
        solid = sim.macros(a)["solid"] == MB_SOLID_SBB
        ux = np.where(solid, 0.0, ux)
        uy = np.where(solid, 0.0, uy)
        F = np.empty((9, A.ny, A.nx))
        uu = ux * ux + uy * uy
        for k in range(9):
            eu = EX[k] * ux + EY[k] * uy
            feq = WK[k] * r * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu)
            q = EX[k] ** 2 * sxx + 2.0 * EX[k] * EY[k] * sxy + EY[k] ** 2 * syy - (sxx + syy) / 3.0
            fneq = np.where(solid, 0.0, -3.0 * WK[k] * r * tau * q)
            F[k] = feq + (1.0 - 1.0 / tau) * fneq
        sim.set_fields(a, r, ux, uy, F, stream)
    sim.sync_history(stream)


def _groups(case_ids, steps_per_d, d_range, bin_width=5.0):
    """Cases grouped by level count and D bin; each group runs
    steps_per_d * (upper edge of its D bin) coarse steps."""
    groups = {}
    for i in case_ids:
        g, prm = batch_case(i, d_range=d_range)
        hi = d_range[0] + bin_width * (np.floor((prm["D"] - d_range[0]) / bin_width) + 1)
        steps = int(steps_per_d * min(hi, d_range[1]))
        groups.setdefault((prm["levels"], steps), []).append((i, g, prm))
    return groups


def generate(case_ids, steps_per_d, precision="f32", h=H, w=W, stream=None, d_range=(10.0, 40.0)):
    """Snapshots of the batched solver: (inputs, targets, masks, kept ids)
    after steps_per_d * D coarse steps from rest (D rounded up to its 5-cell
    bin; the cases of a bin run as one batch); cases whose fields are not
    finite are dropped."""
    xs, ts, ms, ids = [], [], [], []
    for (_, steps), items in _groups(case_ids, steps_per_d, d_range).items():
        sims = []
        for i, g, _ in items:
            s = MultiBlockLBM(g, precision)
            s.init(stream)
            sims.append(s)
        b = Batch(sims)
        b.prepare(steps)
        b.evolution(steps, stream)
        b.close()
        for (i, g, _), s in zip(items, sims):
            if s.check_finite(stream) == 0:
                x, mk = case_inputs(g, h, w)
                t = case_targets(s, g, h, w)
                if np.isfinite(t).all():
                    xs.append(x)
                    ts.append(t)
                    ms.append(mk)
                    ids.append(i)
            s.close()
    return np.stack(xs), np.stack(ts), np.stack(ms), ids


def drag_series(case_ids, steps_per_d, precision, chunk=50, net=None, d_range=(10.0, 40.0), stream=None, kick=0.0):
    """Cd and Cl every `chunk` coarse steps of each case, cold-started (net
    None) or warm-started from the surrogate (with warm_start's kick for
    shedding cases), batched by level count and D bin.  Returns {id: (cd
    series, params, batch key, cl series)} and the device time per coarse
    step of each batch {(levels, steps): ms}."""
    import torch

    out, times = {}, {}
    for key, items in _groups(case_ids, steps_per_d, d_range).items():
        steps = key[1]
        sims = []
        for i, g, _ in items:
            s = MultiBlockLBM(g, precision)
            s.init(stream)
            sims.append(s)
        if net is not None:
            xin = torch.from_numpy(np.stack([case_inputs(g, net.H, net.W)[0] for _, g, _ in items])).cuda()
            pred = predict(net, xin).cpu().numpy()
            for (i, g, _), s, p in zip(items, sims, pred):
                warm_start(s, g, p, stream, kick=kick)
        b = Batch(sims)
        b.prepare(chunk)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms, cds, cls = 0.0, [], []
        for _ in range(steps // chunk):
            e0.record()
            b.evolution(chunk, stream)
            e1.record()
            cd, cl = b.drag(stream)
            ms += e0.elapsed_time(e1)
            cds.append(cd)
            cls.append(cl)
        b.close()
        times[key] = ms / max(1, (steps // chunk) * chunk)
        cds, cls = np.array(cds), np.array(cls)
        for k, (i, g, prm) in enumerate(items):
            out[i] = (cds[:, k], prm, key, cls[:, k])
        for s in sims:
            s.close()
    return out, times


def train(net, x, t, m, epochs, batch=16, lr=1e-3, seed=0, log=None):
    """Adam on mini-batches of the (device) tensors x, t, m; returns the loss
    history (one mean per epoch)."""
    import torch

    rng = np.random.default_rng(seed)
    n = x.shape[0]
    hist = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(x.device)
        tot, cnt = 0.0, 0
        for q in range(0, n - batch + 1, batch):
            idx = perm[q:q + batch]
            xb, tb, mb_ = x[idx].contiguous(), t[idx].contiguous(), m[idx].contiguous()
            tot += net.train_step(xb, tb, mb_, lr)
            cnt += 1
        hist.append(tot / max(cnt, 1))
        if log:
            log(ep, hist[-1])
    return hist


def predict(net, x):
    """Network output (n, h, w, 3) for device inputs x (n, h, w, 4)."""
    import torch

    out = torch.zeros((x.shape[0], x.shape[1], x.shape[2], 3), device=x.device)
    for q in range(0, x.shape[0], net.max_batch):
        xb = x[q:q + net.max_batch].contiguous()
        ob = torch.zeros((xb.shape[0], xb.shape[1], xb.shape[2], 3), device=x.device)
        net.forward(xb, ob)
        out[q:q + xb.shape[0]] = ob
    torch.cuda.synchronize()
    return out


__all__ = ["H", "W", "case_inputs", "case_targets", "coarse_fields", "generate", "predict", "train", "warm_start",
           "updates_per_coarse_step"]
