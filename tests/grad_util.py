"""Per-parameter gradients from the oracle's frame, and the finite-difference
criterion of the reference's gradient check (test infrastructure)."""
import numpy as np

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
SH_C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
         1.445305721320277, -0.5900435899266435]


def sh_basis(dirs, dtu):
    """(N, 15) SH basis values the reference's backward uses (core/cpu/msplat_cpu.cpp:1119-1136)."""
    x, y, z = dirs[:, 0], dirs[:, 1], dirs[:, 2]
    xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
    b = np.zeros((dirs.shape[0], 15))
    if dtu >= 1:
        b[:, 0], b[:, 1], b[:, 2] = -SH_C1 * y, SH_C1 * z, -SH_C1 * x
    if dtu >= 2:
        b[:, 3], b[:, 4], b[:, 5] = SH_C2[0] * xy, SH_C2[1] * yz, SH_C2[2] * (2 * zz - xx - yy)
        b[:, 6], b[:, 7] = SH_C2[3] * xz, SH_C2[4] * (xx - yy)
    if dtu >= 3:
        b[:, 8], b[:, 9] = SH_C3[0] * y * (3 * xx - yy), SH_C3[1] * xy * z
        b[:, 10], b[:, 11] = SH_C3[2] * y * (4 * zz - xx - yy), SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy)
        b[:, 12], b[:, 13] = SH_C3[4] * x * (4 * zz - xx - yy), SH_C3[5] * z * (xx - yy)
        b[:, 14] = SH_C3[6] * x * (xx - 3 * yy)
    return b


def oracle_param_grads(oracle, g, cam, dtu):
    """dL/d(means, scales, quats, dc, rest, opacity logits) of the oracle's last train
    step, from its frame (the SH part through the basis, as the fused Adam uses it)."""
    n = g.n
    vis = oracle.frame("radii") > 0
    v_rgb = oracle.frame("v_rgb").reshape(n, 3).astype(np.float64)
    d = g.means.astype(np.float64) - cam.cam_pos.astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = g.features_rest.shape[1]
    rest = (sh_basis(d, dtu)[:, :k, None] * v_rgb[:, None, :]) * vis[:, None, None]
    dc = SH_C0 * v_rgb * vis[:, None]
    return [oracle.frame("v_mean3d").reshape(n, 3), oracle.frame("v_scale").reshape(n, 3),
            oracle.frame("v_quat").reshape(n, 4), dc, rest, oracle.frame("v_opacity").reshape(n, 1)]


def fd_agreement(analytic, fd, skip=()):
    """The reference's criterion (tests/gradcheck.cpp:354-366): each gradient within 5%
    of its finite difference plus 0.1% of the run's largest gradient. Returns
    (mismatches, checked, cosine)."""
    a = np.concatenate([np.ravel(x) for i, x in enumerate(analytic) if i not in skip]).astype(np.float64)
    f = np.concatenate([np.ravel(x) for i, x in enumerate(fd) if i not in skip]).astype(np.float64)
    gmax = np.abs(a).max()
    bad = np.abs(a - f) > 0.05 * np.maximum(np.abs(a), np.abs(f)) + 1e-3 * gmax
    cos = float(a @ f / np.sqrt((a @ a) * (f @ f) + 1e-300))
    return int(bad.sum()), int(a.size), cos
