"""Numpy restatement of the reference's per-step math (test infrastructure only).

Every function follows one piece of the reference and cites it. With
``dt=np.float32`` the functions keep the reference's FP32 operation order
(including the places where the CUDA C source promotes to double through a
``2.0``/``0.5`` literal); with ``dt=np.float64`` the same formulas run in FP64
and serve as the high-precision twin.

Reference files are cited by their path inside the reference project.
"""
from __future__ import annotations

import numpy as np
import torch

F32, F64 = np.float32, np.float64
PI_LITERAL = 3.14159265359  # NepDescriptorKernels.py:57


def _c(x, dt):
    return np.asarray(x).astype(dt, copy=False)


def _cosf(x, dt):
    """cosf: the argument is rounded to ``dt`` first (a C float parameter)."""
    return np.cos(np.asarray(x).astype(dt).astype(F64)).astype(dt)


def _sinf(x, dt):
    return np.sin(np.asarray(x).astype(dt).astype(F64)).astype(dt)


def _expf(x, dt):
    return np.exp(np.asarray(x).astype(dt).astype(F64)).astype(dt)


# --------------------------------------------------------------------------- pairs
def min_image_filter(pos, nlist, L, cutoff, dt=F32):
    """Minimum image and pair filter of ``DescriptorGenerator.pos_to_pts``
    (``DescriptorGenerator.py:168-182``).

    Returns (index into nlist of kept pairs, kept pairs, translate (P,3)).
    ``translate = pos[j] - pos[i]`` folded once into [-L/2, L/2]; a pair is
    kept when ``|translate| < cutoff`` (compared in double, the cutoff being a
    Python float in the reference).
    """
    pos = _c(pos, dt)
    L = dt(L)
    nl = np.asarray(nlist, np.int64).reshape(-1, 2)
    t = pos[nl[:, 1]] - pos[nl[:, 0]]
    half = dt(0.5) * L
    t = np.where(t > half, t - L, t)
    t = np.where(t < -half, L + t, t)
    d = np.sqrt(t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1] + t[:, 2] * t[:, 2])
    keep = np.nonzero(d.astype(F64) < float(cutoff))[0]
    return keep, nl[keep], t[keep]


def rotate(q, p, trans=None, sign=1, dt=F32):
    """Quaternion rotation of ``get_pts_pairs`` (``PosToPtsKernels.py:54-71``):
    ``a p + 2 (qw (q x p) + (q.p) q) (+/- trans)``, q = (w, x, y, z)."""
    q = _c(q, dt)
    p = _c(p, dt)
    qw, qx, qy, qz = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    px, py, pz = p[..., 0], p[..., 1], p[..., 2]
    a = qw * qw - (qx * qx + qy * qy + qz * qz)
    dot = qx * px + qy * py + qz * pz
    two = dt(2.0)
    ox = a * px + two * (qw * (qy * pz - qz * py) + dot * qx)
    oy = a * py + two * (qw * (qz * px - qx * pz) + dot * qy)
    oz = a * pz + two * (qw * (qx * py - qy * px) + dot * qz)
    out = np.stack([ox, oy, oz], axis=-1)
    if trans is not None:
        t = _c(trans, dt)
        out = out + t if sign > 0 else out - t
    return out


def pair_clouds(quat, pairs, translate, pts_rep, dt=F32):
    """Both point clouds of a pair (``DescriptorGenerator.py:184-218``,
    ``PosToPtsKernels.py:3-150``).

    cloud1: body i at the origin rotated by q_i, then body j rotated by q_j and
    moved by +translate. cloud2: body j at the origin, then body i moved by
    -translate. Shapes (P, 2*npts, 3).
    """
    quat = _c(quat, dt)
    pts = _c(pts_rep, dt)
    qi = quat[pairs[:, 0]][:, None, :]
    qj = quat[pairs[:, 1]][:, None, :]
    t = _c(translate, dt)[:, None, :]
    c1 = np.concatenate([rotate(qi, pts[None], dt=dt), rotate(qj, pts[None], t, +1, dt)], axis=1)
    c2 = np.concatenate([rotate(qj, pts[None], dt=dt), rotate(qi, pts[None], t, -1, dt)], axis=1)
    return c1, c2


def fd_variants(cloud1, cloud2, dx, dteta, dt=F32):
    """The 10 finite-difference clouds (``apply_dx_dteta`` ``PosToPtsKernels.py:153-321``
    and ``apply_dteta2`` ``:324-446``), stacked like ``DescriptorGenerator.py:303``.

    Row ``v*P + p`` is variant v of pair p: v=0 unperturbed; v=1..3 the points
    of body i shifted by +dx along x/y/z; v=4..6 body i rotated by dteta about
    x/y/z (lab axes through the centre of i); v=7..9 body j rotated likewise in
    cloud2. Only the first half of the points (the perturbed body) changes.
    """
    c1 = _c(cloud1, dt)
    c2 = _c(cloud2, dt)
    P, Nd, _ = c1.shape
    h = Nd // 2
    out = np.empty((10, P, Nd, 3), dt)
    for v in range(10):
        base = c1 if v < 7 else c2
        out[v] = base
    dxv = dt(dx)
    for k in range(3):
        out[1 + k, :, :h, k] = c1[:, :h, k] + dxv
    half = dt(dteta) * dt(0.5)
    qw = _cosf(half, dt)
    s = _sinf(half, dt)
    for k in range(3):
        q = np.zeros(4, dt)
        q[0] = qw
        q[1 + k] = s
        out[4 + k, :, :h] = rotate(q, c1[:, :h], dt=dt)
        out[7 + k, :, :h] = rotate(q, c2[:, :h], dt=dt)
    return out.reshape(10 * P, Nd, 3)


# --------------------------------------------------------------------------- descriptor
def radial(pts, nrad, rc, dt=F32):
    """``radial_grad`` (``NepDescriptorKernels.py:3-93``) with its intended
    semantics: centroid over all Nd points (summed in point order), centred
    vectors, Chebyshev radial functions f_n = (1 + T_n(x))/2 * fc and their
    point sums. The kernel's fixed 12-thread block (which drops points >= 12)
    and its missing barrier are not reproduced.

    Returns r (B,Nd,3), |r| (B,Nd), chebo (B,nrad+1,Nd), g_rad (B,nrad+1).
    """
    pts = _c(pts, dt)
    B, Nd, _ = pts.shape
    s = np.zeros((B, 3), dt)
    for a in range(Nd):
        s = s + pts[:, a, :]
    avg = s / dt(Nd)
    r = pts - avg[:, None, :]
    norm = np.sqrt(r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1] + r[..., 2] * r[..., 2])
    u = norm / dt(rc)
    u64 = u.astype(F64)
    x = (2.0 * (u64 - 1.0) * (u64 - 1.0) - 1.0).astype(dt)
    fc = (0.5 * (1.0 + _cosf((PI_LITERAL * u64).astype(dt), dt).astype(F64))).astype(dt)
    fc64 = fc.astype(F64)
    chebo = np.empty((B, nrad + 1, Nd), dt)
    chebo[:, 0] = fc
    if nrad >= 1:
        chebo[:, 1] = ((1.0 + x.astype(F64)) / 2.0 * fc64).astype(dt)
    tm1 = np.ones_like(x)
    tn = x
    for n in range(1, nrad):
        nxt = ((tn * x).astype(F64) * 2.0 - tm1.astype(F64)).astype(dt)
        tm1, tn = tn, nxt
        chebo[:, n + 1] = ((1.0 + nxt.astype(F64)) / 2.0 * fc64).astype(dt)
    g_rad = np.zeros((B, nrad + 1), dt)
    for a in range(Nd):
        g_rad = g_rad + chebo[:, :, a]
    return r, norm, chebo, g_rad


def angular_direct(r, norm, chebo, nang, lmax, dt=F32):
    """O(Nd^2) angular descriptor: ``angular_g`` (``NepDescriptorKernels.py:96-144``)
    for cos(theta_ab) and P_1..P_lmax by recurrence, the outer product of
    ``DescriptorGenerator.py:377`` and the batched matmul of ``:409``.
    g_ang[n*lmax + l-1] = sum_{a,b} f_n(a) f_n(b) P_l(cos theta_ab), diagonal included.
    """
    r = _c(r, dt)
    norm = _c(norm, dt)
    B, Nd, _ = r.shape
    dot = np.zeros((B, Nd, Nd), dt)
    for k in range(3):
        dot = dot + r[:, :, None, k] * r[:, None, :, k]
    dot = dot / (norm[:, :, None] * norm[:, None, :])
    lego = np.empty((B, lmax + 1, Nd * Nd), dt)
    lego[:, 0] = 1
    lego[:, 1] = dot.reshape(B, Nd * Nd)
    flat = lego[:, 1]
    for l in range(1, lmax):
        lego[:, l + 1] = (dt(2.0 * l + 1.0) * flat * lego[:, l] - lego[:, l - 1] * dt(l)) / dt(l + 1)
    # same (transposed-view) operand layout as DescriptorGenerator.py:405-409, so that
    # numpy picks the same BLAS call and summation order as the reference run
    lego_t = lego[:, 1:, :].transpose(0, 2, 1)
    ch = chebo[:, :nang + 1, :]
    outer = (ch[:, :, :, None] * ch[:, :, None, :]).reshape(B, nang + 1, Nd * Nd)
    g_ang = np.matmul(outer, lego_t)
    return g_ang.reshape(B, (nang + 1) * lmax).astype(dt)


def descriptor(pts, hypers, rc, dt=F32, chunk=4096, form="direct"):
    """g_all rows [g_rad (nrad+1) | g_ang ((nang+1)*lmax)] (``DescriptorGenerator.py:432``)."""
    nrad, nang, lmax = (int(h) for h in hypers[:3])
    pts = _c(pts, dt)
    out = []
    for s in range(0, len(pts), chunk):
        r, norm, chebo, g_rad = radial(pts[s:s + chunk], nrad, rc, dt)
        if form == "direct":
            g_ang = angular_direct(r, norm, chebo, nang, lmax, dt)
        else:
            g_ang = angular_sh(r, norm, chebo, nang, lmax, dt)
        out.append(np.concatenate([g_rad, g_ang], axis=1))
    D = (nrad + 1) + (nang + 1) * lmax
    return np.concatenate(out, axis=0) if out else np.zeros((0, D), dt)


def sh_scaled(u, lmax):
    """Real harmonics scaled so that sum_m Y_lm(u) Y_lm(v) = P_l(u.v) for unit
    u, v (Legendre addition theorem), l = 1..lmax, FP64. Order inside each l:
    m = 0, then (cos m, sin m) for m = 1..l. Shape (..., lmax^2 + 2 lmax).

    Y_l0 = P_l(z); Y_lm^{c,s} = sqrt(2 (l-m)!/(l+m)!) Q_l^m(z) {Re,Im}(x+iy)^m,
    Q_l^m = d^m P_l / dz^m from the three-term recurrence of the associated
    Legendre functions.
    """
    from math import factorial, sqrt
    u = np.asarray(u, F64)
    x, y, z = u[..., 0], u[..., 1], u[..., 2]
    C = [np.ones_like(x)]
    S = [np.zeros_like(x)]
    for m in range(1, lmax + 1):
        C.append(x * C[m - 1] - y * S[m - 1])
        S.append(x * S[m - 1] + y * C[m - 1])
    Q = {}
    for m in range(0, lmax + 1):
        dfact = 1.0
        for k in range(1, 2 * m, 2):
            dfact *= k
        Q[(m, m)] = np.full_like(z, dfact)
        if m + 1 <= lmax:
            Q[(m + 1, m)] = (2 * m + 1) * z * Q[(m, m)]
        for l in range(m + 2, lmax + 1):
            Q[(l, m)] = ((2 * l - 1) * z * Q[(l - 1, m)] - (l + m - 1) * Q[(l - 2, m)]) / (l - m)
    cols = []
    for l in range(1, lmax + 1):
        cols.append(Q[(l, 0)])
        for m in range(1, l + 1):
            nrm = sqrt(2.0 * factorial(l - m) / factorial(l + m))
            cols.append(nrm * Q[(l, m)] * C[m])
            cols.append(nrm * Q[(l, m)] * S[m])
    return np.stack(cols, axis=-1)


def angular_sh(r, norm, chebo, nang, lmax, dt=F64):
    """Angular descriptor through the addition theorem:
    sum_{a,b} f_n(a) f_n(b) P_l(rhat_a.rhat_b) = sum_m (sum_a f_n(a) Y_lm(rhat_a))^2.
    Mathematically identical to ``angular_direct``; O(Nd) instead of O(Nd^2)."""
    rh = np.asarray(r, F64) / np.asarray(norm, F64)[..., None]
    Y = sh_scaled(rh, lmax)  # (B, Nd, K)
    f = np.asarray(chebo, F64)[:, :nang + 1, :]  # (B, n, Nd)
    A = np.einsum("bna,bak->bnk", f, Y)
    B = A.shape[0]
    out = np.zeros((B, nang + 1, lmax), F64)
    k = 0
    for l in range(1, lmax + 1):
        out[:, :, l - 1] = np.sum(A[:, :, k:k + 2 * l + 1] ** 2, axis=-1)
        k += 2 * l + 1
    return out.reshape(B, -1).astype(dt)


# --------------------------------------------------------------------------- energy net
def mlp_forward(layers, act, g, dtype=torch.float32):
    """``TheEnergyNet.forward`` (``ForceEvaluator.py:20-26``): Linear + act for
    every layer but the last. ``layers`` = [(W (out,in), b (out,)), ...];
    ``act`` in {"relu", "tanh", "silu"} (the reference uses ReLU)."""
    f = {"relu": torch.relu, "tanh": torch.tanh, "silu": torch.nn.functional.silu}[act]
    h = torch.as_tensor(np.asarray(g)).to(dtype)
    with torch.no_grad():
        for k, (W, b) in enumerate(layers):
            h = torch.nn.functional.linear(h, torch.as_tensor(W).to(dtype), torch.as_tensor(b).to(dtype))
            if k < len(layers) - 1:
                h = f(h)
    return h.numpy()


def fd_forces(e_all, P, dx, dteta, en_min, en_max, dtype=torch.float32):
    """``evaluate_gradients`` + the clip of ``evaluate_forces_torques``
    (``ForceEvaluator.py:86-132``): F = -(e_{1..3}-e_0)/dx, T_i = -(e_{4..6}-e_0)/dteta,
    T_j = -(e_{7..9}-e_0)/dteta, each times (en_max-en_min) and clipped to [-100, 100]."""
    e = torch.as_tensor(np.asarray(e_all)).to(dtype).reshape(10, P)
    e0 = e[0]
    F = torch.stack([-(e[1 + k] - e0) / dx for k in range(3)], dim=1)
    Ti = torch.stack([-(e[4 + k] - e0) / dteta for k in range(3)], dim=1)
    Tj = torch.stack([-(e[7 + k] - e0) / dteta for k in range(3)], dim=1)
    rng = en_max - en_min
    out = []
    for a in (F, Ti, Tj):
        a = a * rng
        a = torch.where(a > 100.0, torch.full_like(a, 100.0), a)
        a = torch.where(a < -100.0, torch.full_like(a, -100.0), a)
        out.append(a.numpy())
    return out


def scatter(pairs, F, Ti, Tj, N, dt=F32):
    """``index_add_`` of ``ForceEvaluator.py:135-142``: F[i] += F, F[j] -= F,
    T[i] += T_i, T[j] += T_j (summed in pair order)."""
    f = np.zeros((N, 3), dt)
    t = np.zeros((N, 3), dt)
    i, j = pairs[:, 0], pairs[:, 1]
    np.add.at(f, i, _c(F, dt))
    np.add.at(f, j, -_c(F, dt))
    np.add.at(t, i, _c(Ti, dt))
    np.add.at(t, j, _c(Tj, dt))
    return f, t


def pair_forces(pos, quat, nlist, L, shape, hypers, layers, act, dx=1e-5, dteta=1e-5,
                dt=F32, form="direct"):
    """Whole force pass of ``Sim.step`` (``Sim.py:261-266``): filter, clouds, 10
    variants, descriptor, net energies, FD forces/torques, scatter.
    Returns dict with pairs, g_all, e_all, F/T per pair and per particle."""
    keep, pairs, t = min_image_filter(pos, nlist, L, shape["cutoff"], dt)
    P = len(pairs)
    c1, c2 = pair_clouds(quat, pairs, t, shape["pts"], dt)
    pts = fd_variants(c1, c2, dx, dteta, dt)
    g = descriptor(pts, hypers, shape["nep_cutoff"], dt, form=form)
    tdt = torch.float32 if dt == F32 else torch.float64
    e = mlp_forward(layers, act, g, tdt)
    Fp, Ti, Tj = fd_forces(e, P, dx, dteta, shape["en_min"], shape["en_max"], tdt)
    N = len(pos)
    Fn, Tn = scatter(pairs, Fp, Ti, Tj, N, dt)
    return dict(keep=keep, pairs=pairs, translate=t, g_all=g, e_all=e.reshape(-1), F_pair=Fp,
                T_i=Ti, T_j=Tj, forces=Fn, torques=Tn, P=P)


# --------------------------------------------------------------------------- integrator
class Thermostat:
    """MTK thermostat state, seeded like ``Sim.setkT`` (``Sim.py:101-105``)."""

    def __init__(self, dt=F32):
        self.var = np.array([-0.0317711, 0.108609, 0.00814227, -0.014238], dt)
        self.thermo_fac = dt(1.00011)


def update_variables(th, N_dof, RN_dof, ke_t, ke_r, timestep, tau, kT, dt=F32):
    """``update_variables`` (``IntegrateStepTwoKernels.py:74-130``)."""
    ts, tau, kT = dt(timestep), dt(tau), dt(kT)
    v0, v1, v2, v3 = (dt(x) for x in th.var)
    c = (ts / tau) / tau
    half = dt(0.5)
    trans_temp = (dt(2.0) / dt(N_dof)) * dt(ke_t)
    xi_p = v0 + half * c * ((trans_temp / kT) - dt(1.0))
    new0 = xi_p + half * c * ((trans_temp / kT) - dt(1.0))
    v1 = v1 + xi_p * ts
    th.thermo_fac = _expf(dt(-0.5) * new0 * ts, dt)
    rot_temp = (dt(2.0) * dt(ke_r)) / dt(RN_dof)
    xi_pr = v2 + half * c * ((rot_temp / kT) - dt(1.0))
    v2n = xi_pr + half * c * ((rot_temp / kT) - dt(1.0))
    v3 = v3 + xi_pr * ts
    th.var = np.array([new0, v1, v2n, v3], dt)


def step_two_rotation(orient, torque, angmom, var2, timestep, dt=F32):
    """``step_two_rotation`` (``IntegrateStepTwoKernels.py:2-71``): torque to the
    body frame, dp = dt * (q-conjugate product), p <- p exp(-dt/2 xi_rot) + dp.
    Returns (new angmom, dp)."""
    o = _c(orient, dt)
    t = _c(torque, dt)
    p = _c(angmom, dt)
    ts = dt(timestep)
    c0, c1, c2, c3 = o[:, 0], -o[:, 1], -o[:, 2], -o[:, 3]
    t1, t2, t3 = t[:, 0], t[:, 1], t[:, 2]
    two = dt(2.0)
    coef1 = c0 * c0 - (c1 * c1 + c2 * c2 + c3 * c3)
    t2x = two * c0 * (c2 * t3 - c3 * t2)
    t2y = two * c0 * (c3 * t1 - c1 * t3)
    t2z = two * c0 * (c1 * t2 - c2 * t1)
    ss = c1 * t1 + c2 * t2 + c3 * t3
    ttx = t1 * coef1 + t2x + two * ss * c1
    tty = t2 * coef1 + t2y + two * ss * c2
    ttz = t3 * coef1 + t2z + two * ss * c3
    dp = np.stack([(c1 * ttx + c2 * tty + c3 * ttz) * ts,
                   ((-c2 * ttz) - (-c3 * tty) + c0 * ttx) * ts,
                   ((-c3 * ttx) - (-c1 * ttz) + c0 * tty) * ts,
                   ((-c1 * tty) - (-c2 * ttx) + c0 * ttz) * ts], axis=1)
    ef = _expf((F64(-ts) / 2.0) * F64(dt(var2)), dt)
    return p * ef + dp, dp


def step_one_translation(pos, vel, accel, thermo_fac, timestep, L, dt=F32):
    """``step_one_translation`` (``IntegrateStepOneKernels.py:185-210``)."""
    pos, vel, accel = _c(pos, dt), _c(vel, dt), _c(accel, dt)
    ts, L, f = dt(timestep), dt(L), dt(thermo_fac)
    nv = (vel + accel * dt(0.5) * ts) * f
    npos = pos + nv * ts
    npos = np.where(npos > dt(0.5) * L, npos - L, npos)
    npos = np.where(npos < -(dt(0.5) * L), npos + L, npos)
    return npos, nv


def _perm(ang, ori, moi_k, scale, ts, which, dt):
    a0, a1, a2, a3 = ang
    o0, o1, o2, o3 = ori
    if which == 1:
        an, on = (-a3, a2, -a1, a0), (-o3, o2, -o1, o0)
    elif which == 2:
        an, on = (-a2, -a3, a0, a1), (-o2, -o3, o0, o1)
    else:
        an, on = (-a1, a0, a3, -a2), (-o1, o0, o3, -o2)
    phi = ((dt(1.0) / dt(4.0)) / dt(moi_k)) * (a0 * on[0] + a1 * on[1] + a2 * on[2] + a3 * on[3])
    arg = (scale * ts) * phi if scale is not None else ts * phi
    cp, sp = _cosf(arg, dt), _sinf(arg, dt)
    ang = tuple(cp * ang[k] + sp * an[k] for k in range(4))
    ori = tuple(cp * ori[k] + sp * on[k] for k in range(4))
    return ang, ori


def step_one_rotation(dp, orient, angmom, var2, timestep, moi, dt=F32):
    """``step_one_rotation`` (``IntegrateStepOneKernels.py:3-182``): kick with dp,
    thermostat factor, then the symmetric free-rotor splitting
    (I_z, dt/2)(I_y, dt/2)(I_x, dt)(I_y, dt/2)(I_z, dt/2) and renormalisation."""
    dp, o, p = _c(dp, dt), _c(orient, dt), _c(angmom, dt)
    ts = dt(timestep)
    ef = _expf((-ts / dt(2.0)) * dt(var2), dt)
    ang = tuple((p[:, k] + dp[:, k]) * ef for k in range(4))
    ori = tuple(o[:, k] for k in range(4))
    h = dt(0.5)
    ang, ori = _perm(ang, ori, moi[2], h, ts, 1, dt)
    ang, ori = _perm(ang, ori, moi[1], h, ts, 2, dt)
    ang, ori = _perm(ang, ori, moi[0], None, ts, 3, dt)
    ang, ori = _perm(ang, ori, moi[1], h, ts, 2, dt)
    ang, ori = _perm(ang, ori, moi[2], h, ts, 1, dt)
    nrm = np.sqrt(ori[0] * ori[0] + ori[1] * ori[1] + ori[2] * ori[2] + ori[3] * ori[3])
    return np.stack([x / nrm for x in ori], axis=1), np.stack(ang, axis=1)


def rot_ke_per_particle(orient, angmom, moi, dt=F32):
    """``rotational_kinetic_energy`` (``IntegrateStepOneKernels.py:213-251``)."""
    o, p = _c(orient, dt), _c(angmom, dt)
    c0, c1, c2, c3 = o[:, 0], -o[:, 1], -o[:, 2], -o[:, 3]
    a0, a1, a2, a3 = p[:, 0], p[:, 1], p[:, 2], p[:, 3]
    sx = ((c0 * a1 + a0 * c1 + (c2 * a3 - c3 * a2)).astype(F64) * 0.5).astype(dt)
    sy = ((c0 * a2 + a0 * c2 + (c3 * a1 - c1 * a3)).astype(F64) * 0.5).astype(dt)
    sz = ((c0 * a3 + a0 * c3 + (c1 * a2 - c2 * a1)).astype(F64) * 0.5).astype(dt)
    m = _c(moi, dt)
    e = (sx * sx) / m[0] + (sy * sy) / m[1] + (sz * sz) / m[2]
    return (e.astype(F64) * 0.5).astype(dt)


class NVTState:
    """Host copy of the simulation state of ``Sim`` (``Sim.py:147-169``)."""

    def __init__(self, pos, vel, orient, angmom, mass, moi, L, kT, timestep, dt=F32,
                 initial_ke_quirk=True):
        self.dt = dt
        self.pos = _c(pos, dt).copy()
        self.vel = _c(vel, dt).copy()
        self.orient = _c(orient, dt).copy()
        self.angmom = _c(angmom, dt).copy()
        self.mass = _c(mass, dt).copy()
        self.moi = _c(moi, dt).copy()
        self.L = dt(L)
        self.kT = dt(kT)
        self.timestep = dt(timestep)
        self.tau = dt(100.0 * timestep)  # Sim.setdt, Sim.py:113-115
        N = len(self.pos)
        self.N_dof = dt((N - 1) * 3)   # Sim.py:35
        self.RN_dof = dt(N * 3)        # Sim.py:36
        self.th = Thermostat(dt)
        ke_t = (dt(0.5) * self.mass) * np.sum(self.vel * self.vel, axis=1)
        # Sim.py:157 keeps the per-particle array; update_variables reads element 0.
        self.ke_t = ke_t[0] if initial_ke_quirk else np.sum(ke_t, dtype=dt)
        self.ke_r = self.initial_rot_ke()
        self.dp = np.zeros_like(self.angmom)
        self.accel = np.zeros_like(self.vel)

    def initial_rot_ke(self):
        """``Sim.getRotKin`` (``Sim.py:171-180``) with ``MathUtils.quaternion_multiplication``."""
        dt = self.dt
        a = self.orient.copy()
        a[:, 1:] = -a[:, 1:]
        b = self.angmom
        vec = (a[:, 0:1] * b[:, 1:] + b[:, 0:1] * a[:, 1:] + np.cross(a[:, 1:], b[:, 1:])) * dt(0.5)
        e = vec[:, 0] * vec[:, 0] / self.moi[0] + vec[:, 1] * vec[:, 1] / self.moi[1] + \
            vec[:, 2] * vec[:, 2] / self.moi[2]
        return np.sum(e * dt(0.5), dtype=dt)

    def step_two(self, forces, torques):
        """``NVT.integrate_step_two`` (``NVT.py:17-64``)."""
        dt = self.dt
        update_variables(self.th, self.N_dof, self.RN_dof, self.ke_t, self.ke_r, self.timestep,
                         self.tau, self.kT, dt)
        self.accel = _c(forces, dt) / self.mass[:, None]
        self.vel = self.vel * self.th.thermo_fac
        self.vel = self.vel + (dt(0.5) * self.timestep) * self.accel
        self.angmom, self.dp = step_two_rotation(self.orient, torques, self.angmom, self.th.var[2],
                                                 self.timestep, dt)

    def step_one(self):
        """``NVT.integrate_step_one`` (``NVT.py:12-15``, ``:67-129``)."""
        dt = self.dt
        self.pos, self.vel = step_one_translation(self.pos, self.vel, self.accel, self.th.thermo_fac,
                                                  self.timestep, self.L, dt)
        self.orient, self.angmom = step_one_rotation(self.dp, self.orient, self.angmom, self.th.var[2],
                                                     self.timestep, self.moi, dt)
        ke = (dt(0.5) * self.mass) * np.sum(self.vel * self.vel, axis=1)
        self.ke_t = np.sum(ke, dtype=dt)
        self.ke_r = np.sum(rot_ke_per_particle(self.orient, self.angmom, self.moi, dt), dtype=dt)
