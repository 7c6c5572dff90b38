"""Float64 restatement of the splatting loss for finite-difference checks (test
infrastructure).

Follows the reference's math (core/cpu/msplat_cpu.cpp): projection with the
1.3 x FOV clamp and 0.3 px EWA dilation (:94-138), pixel centre through the full
projection (:142-146), 3-sigma tile rectangles (:149-157), raw SH colour (:160-190),
front-to-back compositing with the 5.55 / (1/255) / 0.999 / 1e-4 cut-offs
(:574-626), and the zero-padded 11-tap SSIM + L1 loss (:669-785). Everything runs in
float64 and is batched over B parameter sets, so central differences over every
parameter of a small scene are a few batched evaluations.
"""
from __future__ import annotations

import math

import torch

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
SH_C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
         1.445305721320277, -0.5900435899266435]
WIN = [0.0010283801, 0.0075987581, 0.0360007721, 0.1093606895, 0.2130055377, 0.2660117249,
       0.2130055377, 0.1093606895, 0.0360007721, 0.0075987581, 0.0010283801]


def _sh_color(dtu, d, dc, rest):
    """Raw SH colour; d (B,N,3) unit view directions, dc (B,N,3), rest (B,N,K,3)."""
    col = SH_C0 * dc
    if dtu < 1:
        return col
    x, y, z = d[..., 0:1], d[..., 1:2], d[..., 2:3]
    r = rest
    col = col + SH_C1 * (-y * r[:, :, 0] + z * r[:, :, 1] - x * r[:, :, 2])
    if dtu < 2:
        return col
    xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
    col = col + (SH_C2[0] * xy * r[:, :, 3] + SH_C2[1] * yz * r[:, :, 4] + SH_C2[2] * (2 * zz - xx - yy) * r[:, :, 5]
                 + SH_C2[3] * xz * r[:, :, 6] + SH_C2[4] * (xx - yy) * r[:, :, 7])
    if dtu < 3:
        return col
    col = col + (SH_C3[0] * y * (3 * xx - yy) * r[:, :, 8] + SH_C3[1] * xy * z * r[:, :, 9]
                 + SH_C3[2] * y * (4 * zz - xx - yy) * r[:, :, 10] + SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * r[:, :, 11]
                 + SH_C3[4] * x * (4 * zz - xx - yy) * r[:, :, 12] + SH_C3[5] * z * (xx - yy) * r[:, :, 13]
                 + SH_C3[6] * x * (xx - 3 * yy) * r[:, :, 14])
    return col


def _blur(a):
    """Zero-padded separable 11-tap blur of (B, C, H, W)."""
    w = torch.tensor(WIN, dtype=a.dtype, device=a.device)
    b, c, h, wd = a.shape
    x = a.reshape(b * c, 1, h, wd)
    x = torch.nn.functional.conv2d(x, w.view(1, 1, 1, 11), padding=(0, 5))
    x = torch.nn.functional.conv2d(x, w.view(1, 1, 11, 1), padding=(5, 0))
    return x.reshape(b, c, h, wd)


def render_f64(means, scales, quats, dc, rest, opac, cam, bg, dtu):
    """(B, H, W, 3) float64 renders of B parameter sets."""
    dt = torch.float64
    B, N = means.shape[:2]
    W, H = cam.width, cam.height
    vm = torch.as_tensor(cam.viewmat, dtype=dt)
    pm = torch.as_tensor(cam.projmat, dtype=dt)
    pv = means @ vm[:3, :3].T + vm[:3, 3]
    # rotation from the normalised (w, x, y, z) quaternion
    q = quats / quats.norm(dim=-1, keepdim=True)
    w, x, y, z = q.unbind(-1)
    R = torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], -2)
    M = R * torch.exp(scales).unsqueeze(-2)
    cov3 = M @ M.transpose(-1, -2)
    tfx, tfy = 0.5 * W / cam.fx, 0.5 * H / cam.fy
    lx, ly = 1.3 * tfx, 1.3 * tfy
    tz = pv[..., 2]
    tx = tz * torch.clamp(pv[..., 0] / tz, -lx, lx)
    ty = tz * torch.clamp(pv[..., 1] / tz, -ly, ly)
    zero = torch.zeros_like(tz)
    J = torch.stack([torch.stack([cam.fx / tz, zero, -cam.fx * tx / tz ** 2], -1),
                     torch.stack([zero, cam.fy / tz, -cam.fy * ty / tz ** 2], -1)], -2)
    T = J @ vm[:3, :3]
    cov2 = T @ cov3 @ T.transpose(-1, -2) + 0.3 * torch.eye(2, dtype=dt)
    a_, b_, c_ = cov2[..., 0, 0], cov2[..., 0, 1], cov2[..., 1, 1]
    det = a_ * c_ - b_ * b_
    ca, cb, cc = c_ / det, -b_ / det, a_ / det
    ph = torch.cat([means, torch.ones_like(means[..., :1])], -1) @ pm.T
    rw = 1.0 / (ph[..., 3] + 1e-6)
    cxp = 0.5 * W * ph[..., 0] * rw + cam.cx - 0.5
    cyp = 0.5 * H * ph[..., 1] * rw + cam.cy - 0.5
    # 3-sigma tile rectangle (integer, so piecewise constant in the parameters)
    ax = torch.ceil(3 * torch.sqrt(a_))
    ay = torch.ceil(3 * torch.sqrt(c_))
    tx0 = torch.clamp(torch.trunc((cxp - ax) / 16), 0, cam.tiles_x)
    tx1 = torch.clamp(torch.trunc((cxp + ax) / 16 + 1), 0, cam.tiles_x)
    ty0 = torch.clamp(torch.trunc((cyp - ay) / 16), 0, cam.tiles_y)
    ty1 = torch.clamp(torch.trunc((cyp + ay) / 16 + 1), 0, cam.tiles_y)
    visible = (tz > 0.01) & (det != 0) & ((tx1 - tx0) * (ty1 - ty0) > 0)
    cp = torch.as_tensor(cam.cam_pos, dtype=dt)
    d = means - cp
    d = d / d.norm(dim=-1, keepdim=True)
    col = torch.clamp(_sh_color(dtu, d, dc, rest) + 0.5, min=0.0)
    op = torch.sigmoid(opac[..., 0])
    # pixels
    py, px = torch.meshgrid(torch.arange(H, dtype=dt), torch.arange(W, dtype=dt), indexing="ij")
    px, py = px.reshape(-1), py.reshape(-1)
    tile_x, tile_y = torch.div(px, 16, rounding_mode="floor"), torch.div(py, 16, rounding_mode="floor")
    order = torch.argsort(tz, dim=1, stable=True)
    Tr = torch.ones(B, H * W, dtype=dt)
    acc = torch.zeros(B, H * W, 3, dtype=dt)
    done = torch.zeros(B, H * W, dtype=torch.bool)
    bi = torch.arange(B)
    for kk in range(N):
        g = order[:, kk]
        sel = lambda t: t[bi, g]  # noqa: E731
        dx = sel(cxp)[:, None] - px
        dy = sel(cyp)[:, None] - py
        sig = 0.5 * (sel(ca)[:, None] * dx * dx + sel(cc)[:, None] * dy * dy) + sel(cb)[:, None] * dx * dy
        inside = ((tile_x >= sel(tx0)[:, None]) & (tile_x < sel(tx1)[:, None]) & (tile_y >= sel(ty0)[:, None])
                  & (tile_y < sel(ty1)[:, None]) & sel(visible)[:, None])
        ok = inside & (sig >= 0) & (sig < 5.55) & ~done
        alpha = torch.clamp(sel(op)[:, None] * torch.exp(-sig), max=0.999)
        ok = ok & (alpha >= 1.0 / 255.0)
        nT = Tr * (1 - alpha)
        stop = ok & (nT <= 1e-4)
        done = done | stop
        ok = ok & ~stop
        acc = acc + torch.where(ok[..., None], sel(col)[:, None, :] * (alpha * Tr)[..., None], 0.0)
        Tr = torch.where(ok, nT, Tr)
    img = torch.clamp(torch.as_tensor(bg, dtype=dt) * Tr[..., None] + acc, 0.0, 1.0)
    return img.reshape(B, H, W, 3)


def loss_f64(img, gt, ssim_weight):
    """L1 + ssim_weight * (1 - SSIM) per batch element, as msplat_train_step's loss."""
    x = torch.as_tensor(gt, dtype=torch.float64).permute(2, 0, 1).unsqueeze(0).expand(img.shape[0], -1, -1, -1)
    y = img.permute(0, 3, 1, 2)
    mx, my = _blur(x), _blur(y)
    sxx, syy, sxy = _blur(x * x) - mx * mx, _blur(y * y) - my * my, _blur(x * y) - mx * my
    c1, c2 = 0.0001, 0.0009
    ssim = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    per = ssim_weight * (1 - ssim) + (1 - ssim_weight) * (x - y).abs()
    return per.mean(dim=(1, 2, 3))


def finite_differences(params, cam, bg, gt, ssim_weight, dtu, h=1e-4, chunk=256, skip=()):
    """Central differences of the float64 loss w.r.t. every element of the six
    parameter arrays (numpy float32 inputs); returns a list of arrays shaped like them.
    Arrays named in ``skip`` (by index) are left at zero."""
    base = [torch.as_tensor(p, dtype=torch.float64) for p in params]
    sizes = [b.numel() for b in base]
    entries = [(gi, e) for gi, n in enumerate(sizes) if gi not in skip for e in range(n)]
    grads = [torch.zeros(n, dtype=torch.float64) for n in sizes]
    for s in range(0, len(entries), chunk):
        part = entries[s:s + chunk]
        B = 2 * len(part)
        batch = [b.unsqueeze(0).repeat(B, *([1] * b.dim())).reshape(B, -1) for b in base]
        for j, (gi, e) in enumerate(part):
            batch[gi][2 * j, e] += h
            batch[gi][2 * j + 1, e] -= h
        shaped = [bt.reshape((B,) + tuple(b.shape)) for bt, b in zip(batch, base)]
        img = render_f64(*shaped, cam, bg, dtu)
        L = loss_f64(img, gt, ssim_weight)
        for j, (gi, e) in enumerate(part):
            grads[gi][e] = (L[2 * j] - L[2 * j + 1]) / (2 * h)
    return [g.reshape(b.shape).numpy() for g, b in zip(grads, base)]
