"""The reduced radial tensor R: its inputs (the reference's MATLAB driver, restated) and the GPU
quadrature.

``sumfac_inputs`` restates src/GeneralCollisionTensor.m:43-181, which prepares the 26 inputs of the
reference's ``compute_rtensor_sumfac_mex`` -- grid sizes from the paddings (:54-64), Gauss rules
(:66-79), radial and angular normalisations (:81-104), the l-triplet table, the valid-q_i lists and
the P_gain / P_loss tables (:106-174); ``conservation_zero`` is the rule of :183-191 that zeroes
the rows of R feeding mass, momentum and energy.  ``compute_R`` runs the quadrature on the GPU
(cf_rtensor_sumfac) from those inputs.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib, basis, quadrature
from .geometry import Geometry


def grid_sizes(K_max: int, L_max: int, radial_pad: int, angular_pad: int) -> dict:
    """Quadrature sizes of src/GeneralCollisionTensor.m:55-64."""
    return dict(
        N_x=radial_pad + math.ceil((3 * K_max + 1.5 * L_max + 3) / 2.0),
        N_u1=radial_pad + 4 * K_max + 3 * L_max + 4,
        N_t1=angular_pad + K_max + math.ceil(1.5 * L_max) + 1,
        N_y2=angular_pad + 4 * K_max + 3 * L_max + 4,
        N_t2=radial_pad + 3 * K_max + math.floor(1.5 * L_max) + 3,
        N_chi=K_max + math.ceil(0.5 * L_max) + 1,
        N_eps=2 * K_max + L_max + 1,
    )


def sumfac_inputs(geo: Geometry, K_max: int, gamma: float, radial_pad: int = 40, angular_pad: int = 0,
                  packed: bool = False):
    """The 26 MEX inputs, in order (src/GeneralCollisionTensor.m:177-181).

    ``geo`` must be in the reference's unsorted (find) order: the first entry of
    each l-triplet decides that triplet's (l_i, l_j, l_k) and q_i lists are built
    in entry order (:116-173).

    With ``packed``, returns ``(args, pg1, pg2)``: the two gain tables (inputs 24 and 26) come
    compressed to the valid (q_i, channel) pairs, in the layout cf_rtensor_sumfac_packed takes
    (``pg1[u, t, j]``, ``pg2[y, j]``, C order), and are left empty in ``args``.  The compressed
    values are the dense tables' own, summed in the same order.
    """
    L = geo.L
    N_K = K_max + 1
    NQ = basis.n_q(L)
    s = grid_sizes(K_max, L, radial_pad, angular_pad)
    qx = quadrature.generalized_laguerre(s["N_x"], gamma / 2.0)
    qu1 = quadrature.legendre(s["N_u1"], 0.0, 1.0)
    qt1 = quadrature.legendre(s["N_t1"], 0.0, 1.0)
    qy2 = quadrature.legendre(s["N_y2"], 0.0, 1.0)
    qt2 = quadrature.legendre(s["N_t2"], 0.0, 1.0)
    qchi = quadrature.legendre(s["N_chi"], -1.0, 1.0)
    N_eps = s["N_eps"]
    eps_vec = 2.0 * math.pi * np.arange(N_eps) / N_eps
    W_eps = (2.0 * math.pi / N_eps) * np.ones(N_eps)

    radial_norm = np.array([[basis.radial_norm(k, l) for l in range(L + 1)] for k in range(N_K)])
    sh_norm = np.zeros(NQ)
    for l in range(L + 1):
        for m in range(-l, l + 1):
            sh_norm[basis.q_index(l, m) - 1] = basis.sh_norm(l, m)

    N_L = int(np.max(geo.ic_map))
    N_t1, N_u1, N_y2 = s["N_t1"], s["N_u1"], s["N_y2"]
    L_triplets = np.zeros((N_L, 3))
    qi_valid = -np.ones((NQ, N_L))
    P_loss_p1 = np.zeros((N_t1, N_u1, N_L))
    P_loss_p2 = np.zeros((N_y2, N_L))
    if packed:
        P_gain_p1 = P_gain_p2 = None
        cols1: list[np.ndarray] = []  # per channel [n_qi, N_t1, N_u1]
        cols2: list[np.ndarray] = []  # per channel [n_qi, N_y2]
    else:
        P_gain_p1 = np.zeros((N_t1, N_u1, NQ, N_L))
        P_gain_p2 = np.zeros((N_y2, NQ, N_L))

    # SH values at phi = 0 on the two patches' polar grids (:143-145, :156-158)
    y1 = qu1.x[None, :] * qt1.x[:, None]  # [N_t1, N_u1]
    mu1 = np.clip(1.0 - 2.0 * y1**2, -1.0, 1.0)
    Y1 = basis.real_sh(L, np.arccos(mu1).ravel(), np.zeros(mu1.size)).reshape(N_t1, N_u1, NQ)
    mu2 = np.clip(1.0 - 2.0 * qy2.x**2, -1.0, 1.0)
    Y2 = basis.real_sh(L, np.arccos(mu2), np.zeros(N_y2))  # [N_y2, NQ]
    if packed:
        Y1q = np.ascontiguousarray(Y1.transpose(2, 0, 1))  # [NQ, N_t1, N_u1]: the same values, q-major
        Y2q = np.ascontiguousarray(Y2.T)  # [NQ, N_y2]

    labels = geo.labels.astype(np.int64)
    ic = geo.ic_map.astype(np.int64)
    order = np.argsort(ic, kind="stable")
    bounds = np.searchsorted(ic[order], np.arange(1, N_L + 2))
    for t in range(N_L):
        g_idx = order[bounds[t]:bounds[t + 1]]
        first = labels[g_idx[0]]
        l_i, l_j, l_k = (int(math.floor(math.sqrt(q - 1))) for q in first)
        L_triplets[t] = (l_i, l_j, l_k)
        q_i0 = l_i * l_i + l_i + 1
        q_j0 = l_j * l_j + l_j + 1
        Y_i0 = math.sqrt((2 * l_i + 1) / (4.0 * math.pi))
        Y_j0 = math.sqrt((2 * l_j + 1) / (4.0 * math.pi))
        D_full = float(np.sum(geo.vals[g_idx] ** 2))
        scale = (8.0 * math.pi**2 * Y_j0) / D_full
        qi_list: list[int] = []
        if packed:
            c1: list[np.ndarray] = []
            c2: list[np.ndarray] = []
        for g in g_idx:
            q_i, q_j, q_k = (int(v) for v in labels[g])
            if q_j != q_j0:
                continue
            G = float(geo.vals[g])
            if q_i not in qi_list:
                qi_list.append(q_i)
                if packed:
                    c1.append(np.zeros((N_t1, N_u1)))
                    c2.append(np.zeros(N_y2))
            if packed:
                j = qi_list.index(q_i)
                c1[j] += G * Y1q[q_k - 1]
                c2[j] += G * Y2q[q_k - 1]
            else:
                P_gain_p1[:, :, q_i - 1, t] += G * Y1[:, :, q_k - 1]
                P_gain_p2[:, q_i - 1, t] += G * Y2[:, q_k - 1]
            if q_i == q_i0:
                P_loss_p1[:, :, t] += G * Y_i0 * Y1[:, :, q_k - 1]
                P_loss_p2[:, t] += G * Y_i0 * Y2[:, q_k - 1]
        if packed:
            for j in range(len(qi_list)):
                c1[j] *= scale
                c2[j] *= scale
            cols1.append(np.stack(c1) if c1 else np.zeros((0, N_t1, N_u1)))
            cols2.append(np.stack(c2) if c2 else np.zeros((0, N_y2)))
        else:
            P_gain_p1[:, :, :, t] *= scale
            P_gain_p2[:, :, t] *= scale
        P_loss_p1[:, :, t] *= scale
        P_loss_p2[:, t] *= scale
        qi_valid[: len(qi_list), t] = qi_list

    col = lambda a: np.asarray(a, dtype=np.float64).reshape(-1, 1)  # noqa: E731
    args = [
        float(K_max), float(N_L), float(NQ), float(gamma),
        col(qx.x), col(qx.w), col(qu1.x), col(qu1.w), col(qt1.x), col(qt1.w),
        col(qy2.x), col(qy2.w), col(qt2.x), col(qt2.w), col(qchi.x), col(qchi.w), col(eps_vec), col(W_eps),
        radial_norm, col(sh_norm), L_triplets, qi_valid,
        P_loss_p1, P_gain_p1, P_loss_p2, P_gain_p2,
    ]
    if not packed:
        return args
    nnz = sum(c.shape[0] for c in cols1)
    pg1 = np.empty((N_u1, N_t1, nnz))
    pg2 = np.empty((N_y2, nnz))
    j0 = 0
    for c1, c2 in zip(cols1, cols2):
        n = c1.shape[0]
        pg1[:, :, j0:j0 + n] = c1.transpose(2, 1, 0)
        pg2[:, j0:j0 + n] = c2.T
        j0 += n
    args[23] = np.zeros(0)
    args[25] = np.zeros(0)
    return args, pg1, pg2


def conservation_zero(R: np.ndarray, L_triplets: np.ndarray) -> np.ndarray:
    """Zero R rows k1 = 0, 1 for l_i = 0 and k1 = 0 for l_i = 1 (src/GeneralCollisionTensor.m:184-191)."""
    R = R.copy(order="F")
    for t in range(L_triplets.shape[0]):
        li = int(L_triplets[t, 0])
        if li == 0:
            R[0, :, :, t] = 0.0
            if R.shape[0] > 1:
                R[1, :, :, t] = 0.0
        elif li == 1:
            R[0, :, :, t] = 0.0
    return R


def l_triplets_of(geo: Geometry) -> np.ndarray:
    """(l_i, l_j, l_k) of each ic_map channel, taken from its first entry (src/GeneralCollisionTensor.m:117-122)."""
    N_L = int(np.max(geo.ic_map))
    out = np.zeros((N_L, 3), dtype=np.int64)
    seen = np.zeros(N_L, dtype=bool)
    for z in range(geo.n_g):
        t = int(geo.ic_map[z]) - 1
        if not seen[t]:
            seen[t] = True
            out[t] = np.floor(np.sqrt(geo.labels[z] - 1.0)).astype(np.int64)
    return out



def compute_R(args: list, device: int = 0, zero_conservation: bool = True, timing: dict | None = None,
              packed: tuple | None = None) -> np.ndarray:
    """R [K x K x K x N_L] (Fortran order) from the 26 sumfac inputs, on the GPU.

    ``args`` is the input list of compute_rtensor_sumfac_mex (``sumfac_inputs``); the result is the
    quadrature, with the conservation rows zeroed as the MATLAB driver does unless
    ``zero_conservation`` is False (then it is the MEX output itself).  ``packed`` = (pg1, pg2), the
    compressed gain tables of ``sumfac_inputs(..., packed=True)``, runs cf_rtensor_sumfac_packed
    instead (the dense tables in ``args`` are then ignored).  ``timing``, if given, receives the
    device seconds of the quadrature kernels."""
    D = C.POINTER(C.c_double)
    keep = [np.ascontiguousarray(np.asarray(a if a is not None else np.zeros(0), dtype=np.float64).ravel(order="F"))
            for a in args[4:]]
    p = [a.ctypes.data_as(D) for a in keep]
    n = [a.size for a in keep]
    K_max, N_L, N_Q = int(args[0]), int(args[1]), int(args[2])
    inp = _lib.SumfacInputs(K_max, N_L, N_Q, float(args[3]),
                            p[0], p[1], n[0], p[2], p[3], n[2], p[4], p[5], n[4], p[6], p[7], n[6],
                            p[8], p[9], n[8], p[10], p[11], n[10], p[12], p[13], n[12],
                            p[14], p[15], p[16], p[17], p[18], p[19], p[20], p[21])
    N_K = K_max + 1
    R = np.zeros(N_K**3 * N_L)
    dev_s = C.c_double(0.0)
    lib = _lib.load()
    if packed is not None:
        pg1 = np.ascontiguousarray(packed[0], dtype=np.float64)
        pg2 = np.ascontiguousarray(packed[1], dtype=np.float64)
        _lib.check(lib.cf_rtensor_sumfac_packed(R.ctypes.data_as(D), C.byref(inp), pg1.ctypes.data_as(D),
                                                pg2.ctypes.data_as(D), int(device), C.byref(dev_s)))
    else:
        _lib.check(lib.cf_rtensor_sumfac(R.ctypes.data_as(D), C.byref(inp), int(device), C.byref(dev_s)))
    if timing is not None:
        timing["device_seconds"] = dev_s.value
    R = np.asfortranarray(R.reshape(N_K, N_K, N_K, N_L, order="F"))
    return conservation_zero(R, np.asarray(args[20])) if zero_conservation else R


def hard_sphere_R(L: int, K_max: int, pad: int = 20, device: int = 0, timing: dict | None = None) -> np.ndarray:
    """Hard-sphere (gamma = 1) R at (L, K_max) with radial and angular pad ``pad``, on the GPU, from
    the compressed gain tables (the route that fits host memory at L = 16)."""
    from .geometry import generate_geometry

    geo = generate_geometry(L)
    args, pg1, pg2 = sumfac_inputs(geo, K_max, 1.0, pad, pad, packed=True)
    return compute_R(args, device=device, timing=timing, packed=(pg1, pg2))
