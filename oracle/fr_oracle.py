"""CPU oracle for the explicit FR residual-and-update path.

TEST INFRASTRUCTURE ONLY.  This is a numpy restatement of the reference
(AutoFlowCFD) algorithm, used by ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` to check results.  The product path
(``autoflowcfd_b200``) never imports it.

It is pinned against the golden fixtures in ``tests/golden`` that the
reference itself produced (``tests/golden/make_golden.py``); see
``tests/test_oracle_golden.py``.

Every function cites the reference file:line it restates (paths are relative
to the reference's ``src/autoflowcfd``).  Inputs are the flattened arrays the
reference feeds its Numba kernels (``core/fr_operators/face_kernels.py:124-187``)
plus the Jacobians and operators, as stored in a ``case`` mapping:

    case["det_jacs"] (N,S)          case["inv_jacs"] (N,S,3,3)
    case["det_jacs_fine"] (N,Fn)    case["inv_jacs_fine"] (N,Fn,3,3)
    case["D_3d_prism"/"_tet"] (S,S,3), c2f/Dfine/f2c_{prism,tet}, filter_{prism,tet}
    face tables: owner_cell ... colors (see make_golden.flat_tables)
    boundary tables: bc_group, bc_type, bc_noslip, bc_wall_vel, bc_Q, bc_p_out
"""

from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

GAMMA = 1.4
R_AIR = 287.0
PR = 0.72
PR_T = 0.9
C_IP = 4.0
OUTLIER_FACTOR = 1e4
OUTLIER_FIELD_FLOOR = 1e-9
BC_WALL, BC_FARFIELD, BC_INLET, BC_OUTLET, BC_SYMMETRY = 0, 1, 2, 3, 4

# SST constants, core/turbulence/sst.py:52-63, 187
SST = dict(sigma_k1=0.85, sigma_k2=1.0, sigma_w1=0.5, sigma_w2=0.856, beta1=0.075, beta2=0.0828,
           a1=0.31, kappa=0.41, beta_star=0.09, tvr_max=1.0e5)
MU_SST_SOURCE = 1.8e-5  # core/fr_solver/turbulence.py:230


# ---------------------------------------------------------------------------
# pointwise physics
# ---------------------------------------------------------------------------
def conserved_to_primitive(U5):
    """core/fr_residual/inviscid.py:38-47 (rho >= 1e-10, no pressure floor)."""
    rho = np.maximum(U5[..., 0], 1e-10)
    u = U5[..., 1] / rho
    v = U5[..., 2] / rho
    w = U5[..., 3] / rho
    E = U5[..., 4] / rho
    ke = 0.5 * (u**2 + v**2 + w**2)
    p = (GAMMA - 1.0) * rho * (E - ke)
    return np.stack([rho, u, v, w, p], axis=-1)


def state_primitives(U):
    """FRState._update_primitives, core/fr_solver/state.py:76-97 (p >= 1)."""
    rho = np.maximum(U[..., 0], 1e-10)
    u = U[..., 1] / rho
    v = U[..., 2] / rho
    w = U[..., 3] / rho
    ke = 0.5 * (u**2 + v**2 + w**2)
    p = np.maximum((U[..., 4] - rho * ke) * 0.4, 1.0)
    Q = np.zeros_like(U)
    Q[..., 0], Q[..., 1], Q[..., 2], Q[..., 3], Q[..., 4] = rho, u, v, w, p
    if U.shape[-1] > 5:
        Q[..., 5] = np.maximum(U[..., 5] / rho, 1e-12)
        Q[..., 6] = np.maximum(U[..., 6] / rho, 1e-12)
    return Q


def euler_flux(Q):
    """euler_physical_flux_point, core/fr_operators/flux_kernels.py:28-68 -> (...,3,5)."""
    rho, u, v, w, p = (Q[..., i] for i in range(5))
    rs = np.maximum(rho, 1e-10)
    ke = 0.5 * (u * u + v * v + w * w)
    e_int = p / ((GAMMA - 1.0) * rs)
    rhoE = rho * (e_int + ke)
    H = (rhoE + p) / rs
    mf = (rho * u, rho * v, rho * w)
    vel = (u, v, w)
    F = np.zeros(Q.shape[:-1] + (3, 5))
    for i in range(3):
        F[..., i, 0] = mf[i]
        F[..., i, 1] = mf[i] * u + (p if i == 0 else 0.0)
        F[..., i, 2] = mf[i] * v + (p if i == 1 else 0.0)
        F[..., i, 3] = mf[i] * w + (p if i == 2 else 0.0)
        F[..., i, 4] = rho * H * vel[i]
    return F


def ausm_up(qL, qR, n):
    """compute_ausm_up_flux, core/fr_operators/kernels.py:19-155, vectorised over leading axes."""
    alpha, beta, Kp, Ku, sigma_p, ma_ref = 0.1875, 0.5, 0.25, 0.75, 1.0, 0.1
    rhoL = np.maximum(qL[..., 0], 1e-6)
    rhoR = np.maximum(qR[..., 0], 1e-6)
    pL = np.maximum(qL[..., 4], 10.0)
    pR = np.maximum(qR[..., 4], 10.0)
    uL, vL, wL = qL[..., 1], qL[..., 2], qL[..., 3]
    uR, vR, wR = qR[..., 1], qR[..., 2], qR[..., 3]
    nx, ny, nz = n[..., 0], n[..., 1], n[..., 2]
    unL = uL * nx + vL * ny + wL * nz
    unR = uR * nx + vR * ny + wR * nz
    aL = np.sqrt(np.maximum(GAMMA * pL / rhoL, 1e-10))
    aR = np.sqrt(np.maximum(GAMMA * pR / rhoR, 1e-10))
    ML = unL / np.maximum(aL, 1e-10)
    MR = unR / np.maximum(aR, 1e-10)
    a_half = 0.5 * (aL + aR)
    rho_half = 0.5 * (rhoL + rhoR)
    Mbar2 = (unL**2 + unR**2) / (2.0 * a_half**2)
    M0 = np.minimum(1.0, np.maximum(Mbar2, ma_ref**2))
    fa = np.sqrt(M0) * (2.0 - np.sqrt(M0))
    fa = np.maximum(fa, 1e-6)

    def m_plus(M):
        return np.where(np.abs(M) >= 1, 0.5 * (M + np.abs(M)), 0.25 * (M + 1) ** 2 + alpha * (M**2 - 1) ** 2)

    def m_minus(M):
        return np.where(np.abs(M) >= 1, 0.5 * (M - np.abs(M)), -0.25 * (M - 1) ** 2 - alpha * (M**2 - 1) ** 2)

    def p_plus(M):
        return np.where(np.abs(M) >= 1, 0.5 * (1 + np.sign(M)),
                        0.25 * ((M + 1) ** 2 * (2 - M) + beta * M * (M**2 - 1) ** 2))

    def p_minus(M):
        return np.where(np.abs(M) >= 1, 0.5 * (1 - np.sign(M)),
                        0.25 * ((M - 1) ** 2 * (2 + M) - beta * M * (M**2 - 1) ** 2))

    M_half = m_plus(ML) + m_minus(MR)
    Mp = -(Kp / fa) * np.maximum(1.0 - sigma_p * Mbar2, 0.0) * (pR - pL) / (rho_half * a_half**2)
    mdot = 0.5 * (rhoL * aL + rhoR * aR) * (M_half + Mp)
    PpL = p_plus(ML)
    PmR = p_minus(MR)
    p_half = PpL * pL + PmR * pR - Ku * PpL * PmR * (rhoL + rhoR) * fa * a_half * (unR - unL)
    up = mdot >= 0.0
    out = np.empty(qL.shape[:-1] + (5,))
    out[..., 0] = mdot
    out[..., 1] = mdot * np.where(up, uL, uR) + p_half * nx
    out[..., 2] = mdot * np.where(up, vL, vR) + p_half * ny
    out[..., 3] = mdot * np.where(up, wL, wR) + p_half * nz
    hL = GAMMA / (GAMMA - 1) * pL / rhoL + 0.5 * (uL**2 + vL**2 + wL**2)
    hR = GAMMA / (GAMMA - 1) * pR / rhoR + 0.5 * (uR**2 + vR**2 + wR**2)
    out[..., 4] = mdot * np.where(up, hL, hR)
    return out


def viscous_flux(Q, gv, gT, mu, mu_t):
    """viscous_physical_flux_point, core/fr_operators/flux_kernels.py:71-137 -> (...,3,5)."""
    mt = mu + mu_t
    S00, S11, S22 = gv[..., 0, 0], gv[..., 1, 1], gv[..., 2, 2]
    S01 = 0.5 * (gv[..., 0, 1] + gv[..., 1, 0])
    S02 = 0.5 * (gv[..., 0, 2] + gv[..., 2, 0])
    S12 = 0.5 * (gv[..., 1, 2] + gv[..., 2, 1])
    div = gv[..., 0, 0] + gv[..., 1, 1] + gv[..., 2, 2]
    lam = -2.0 / 3.0 * mt
    t00 = 2.0 * mt * S00 + lam * div
    t11 = 2.0 * mt * S11 + lam * div
    t22 = 2.0 * mt * S22 + lam * div
    t01 = 2.0 * mt * S01
    t02 = 2.0 * mt * S02
    t12 = 2.0 * mt * S12
    cp = GAMMA * R_AIR / (GAMMA - 1.0)
    k = mu * cp / PR + mu_t * cp / PR_T
    u, v, w = Q[..., 1], Q[..., 2], Q[..., 3]
    G = np.zeros(Q.shape[:-1] + (3, 5))
    G[..., 0, 1], G[..., 0, 2], G[..., 0, 3] = t00, t01, t02
    G[..., 1, 1], G[..., 1, 2], G[..., 1, 3] = t01, t11, t12
    G[..., 2, 1], G[..., 2, 2], G[..., 2, 3] = t02, t12, t22
    G[..., 0, 4] = (u * t00 + v * t01 + w * t02) + (-k * gT[..., 0])
    G[..., 1, 4] = (u * t01 + v * t11 + w * t12) + (-k * gT[..., 1])
    G[..., 2, 4] = (u * t02 + v * t12 + w * t22) + (-k * gT[..., 2])
    return G


# ---------------------------------------------------------------------------
# mesh-level helpers
# ---------------------------------------------------------------------------
@dataclass
class Mesh:
    """Arrays of one case, with derived per-cell-type operator views."""

    c: Dict[str, np.ndarray]
    N: int = 0
    S: int = 0
    n_prism: int = 0
    order: int = 0
    extras: Dict[str, np.ndarray] = field(default_factory=dict)

    @classmethod
    def from_case(cls, case):
        c = {k: case[k] for k in case.keys()}
        m = cls(c=c, N=int(c["n_cells"]), S=int(c["n_sps"]), n_prism=int(c["n_prism"]), order=int(c["order"]))
        det = c["det_jacs"]
        m.extras["adj"] = det[..., None, None] * c["inv_jacs"]  # compute_adj_j, volume_contract.py:47-80
        m.extras["adj_fine"] = c["det_jacs_fine"][..., None, None] * c["inv_jacs_fine"]
        return m

    def split(self):
        """(slice, suffix) for the prism and tet blocks."""
        out = []
        if self.n_prism > 0:
            out.append((slice(0, self.n_prism), "prism"))
        if self.N > self.n_prism:
            out.append((slice(self.n_prism, self.N), "tet"))
        return out


def contract_1axis(D, X):
    """contract_shared_operator_1axis, core/fr_operators/volume_contract.py:83-96."""
    return np.matmul(D, X)


def contract_2axis(D, X):
    """contract_shared_operator_2axis, core/fr_operators/volume_contract.py:99-113."""
    F, J, M = D.shape
    return np.matmul(D.reshape(F, J * M), X.reshape(X.shape[0], J * M, X.shape[-1]))


def physical_gradient(m: Mesh, field_):
    """compute_physical_gradient, core/fr_operators/gradients.py:23-64 -> (N,S,nf,3)."""
    N, S, nf = field_.shape
    grad_comp = np.zeros((N, S, 3, nf))
    for sl, t in m.split():
        D = m.c["D_3d_" + t]
        D2 = np.ascontiguousarray(np.transpose(D, (0, 2, 1))).reshape(S * 3, S)
        n = sl.stop - sl.start
        grad_comp[sl] = contract_1axis(D2, field_[sl]).reshape(n, S, 3, nf)
    return np.matmul(np.swapaxes(grad_comp, -1, -2), m.c["inv_jacs"])


def suppress_outliers(R, ref):
    """suppress_residual_outliers, core/fr_operators/troubled_cell.py:346-408."""
    med = np.median(np.abs(R), axis=1)[:, None, :]
    ref_field = OUTLIER_FIELD_FLOOR * np.mean(np.abs(ref), axis=1, keepdims=True)
    thr = np.maximum(np.maximum(med, ref_field), 1e-300)
    out = np.abs(R) > OUTLIER_FACTOR * thr
    if not np.any(out):
        return R
    return np.where(out, 0.0, R)


def extrap_E(m: Mesh, cells, axis, side):
    """boundary_extrap[celltype, axis, side_idx] per face -> (F,P,S)."""
    ct = (cells >= m.n_prism).astype(np.int64)
    si = np.where(side < 0, 0, 1)
    return m.c["boundary_extrap"][ct, axis, si]


def distribute(m: Mesh, jump, axis, side):
    """_distribute_point, core/fr_residual/inviscid_kernel_colored.py:28-40:
    contrib[s] = g'[coord(s)] * jump[fp(s)] with g' = g_left for side<0."""
    fp = m.c["dist_fp_of_sp"][axis]  # (F,S)
    co = m.c["dist_axis_coord_of_sp"][axis]
    g = np.where((side < 0)[:, None], m.c["g_left"][co], m.c["g_right"][co])
    jf = np.take_along_axis(jump, fp[..., None], axis=1)  # (F,S,V)
    return g[..., None] * jf


def gather_sources(m: Mesh, f, field_, which):
    """Neighbour-side assembly sum_k src_k @ field[cell_k], inviscid_kernel_colored.py:112-130."""
    c0 = m.c[which + "_src0_cell"][f]
    mat0 = m.c[which + "_src0_mat"][f]
    nf = field_.shape[-1]
    out = np.zeros((len(f), mat0.shape[1], nf))
    ok = c0 >= 0
    out[ok] = np.matmul(mat0[ok], field_[c0[ok]])
    i1 = m.c[which + "_src1_idx"][f]
    has1 = i1 >= 0
    if np.any(has1):
        c1 = m.c[which + "_src1_cell"][i1[has1]]
        mat1 = m.c[which + "_src1_mat"][i1[has1]]
        out[has1] = out[has1] + np.matmul(mat1, field_[c1])
    return out


def ghost_states(m: Mesh, Q, faces):
    """compute_boundary_ghost_states + BoundaryGhostStateProvider,
    core/fr_residual/inviscid_kernel.py:288-310, boundary/fr_ghost_state.py:26-189."""
    oc = m.c["owner_cell"][faces]
    E = extrap_E(m, oc, m.c["owner_axis"][faces], m.c["owner_side"][faces])
    Qo = np.matmul(E, Q[oc])  # (F,P,5)
    n = m.c["true_normal"][faces]
    code = m.c["bc_group"][faces]
    typ = m.c["bc_type"][code]
    G = Qo.copy()
    vn = np.sum(Qo[..., 1:4] * n, axis=-1)
    # WALL no-slip: 2 v_w - v ; slip: reflect
    wall = typ == BC_WALL
    noslip = wall & (m.c["bc_noslip"][code] == 1)
    slip = wall & ~noslip
    vw = m.c["bc_wall_vel"][code]
    G[noslip, :, 1:4] = 2.0 * vw[noslip][:, None, :] - Qo[noslip, :, 1:4]
    refl = Qo[..., 1:4] - 2.0 * vn[..., None] * n
    G[slip, :, 1:4] = refl[slip]
    far = typ == BC_FARFIELD
    G[far] = m.c["bc_Q"][code[far]][:, None, :]
    inl = typ == BC_INLET
    inflow = (vn < 0.0) & inl[:, None]
    Qin = np.broadcast_to(m.c["bc_Q"][code][:, None, :], Qo.shape)
    G = np.where(inflow[..., None], Qin, G)
    outl = typ == BC_OUTLET
    outflow = (vn > 0.0) & outl[:, None]
    pout = np.broadcast_to(m.c["bc_p_out"][code][:, None], vn.shape)
    G[..., 4] = np.where(outflow, pout, G[..., 4])
    sym = typ == BC_SYMMETRY
    G[sym, :, 1:4] = refl[sym]
    return Qo, G


def greedy_face_coloring(owner, neighbor, is_boundary, n_cells):
    """greedy_face_coloring, core/utils/face_coloring.py:124-176: faces in order,
    each takes the smallest color no earlier face sharing one of its cells
    (the owner, and the neighbour of an interior face) already has."""
    owner = np.asarray(owner, np.int64)
    nb = np.where(np.asarray(is_boundary).astype(bool), -1, np.asarray(neighbor, np.int64))
    cell_faces = [[] for _ in range(int(n_cells))]
    for f in range(len(owner)):
        cell_faces[owner[f]].append(f)
        if nb[f] >= 0:
            cell_faces[nb[f]].append(f)
    colors = np.full(len(owner), -1, np.int32)
    for f in range(len(owner)):
        used = set()
        for c in (owner[f], nb[f]):
            if c >= 0:
                used.update(int(colors[g]) for g in cell_faces[c] if g != f and colors[g] >= 0)
        k = 0
        while k in used:
            k += 1
        colors[f] = k
    return colors


def _color_faces(m: Mesh):
    col = m.c["colors"]
    return [np.flatnonzero(col == c) for c in range(int(col.max()) + 1)]


# ---------------------------------------------------------------------------
# residuals
# ---------------------------------------------------------------------------
def inviscid_residual_p0(m: Mesh, U):
    """compute_inviscid_residual_fv_p0, core/fr_residual/inviscid_p0.py:18-85 with
    the kernel core/fr_residual/inviscid_p0_kernel.py:25-108: finite volume at
    order 0 -- per face record, AUSM+up between the owner's and the
    neighbour's (or ghost) state along the unit normal, times the face area,
    taken out of the owner and added to the neighbour (divided by the cell
    volumes); no primary-flag filtering.  Faces are added in record order."""
    N = m.N
    Q = conserved_to_primitive(U[..., :5])[:, 0, :]
    isb = m.c["is_boundary"].astype(bool)
    own, nbr = m.c["owner_cell"], m.c["neighbor_cell"]
    n = m.c["true_normal"][:, 0, :]
    area = m.c["true_area_weight"][:, 0]
    # mesh.cell_volumes: computed at the order the mesh was loaded at (the
    # target order during an order continuation), not the current order's
    vol = m.c["fv_cell_volumes"] if "fv_cell_volumes" in m.c else m.c["cell_volumes"]
    Qn = Q[np.where(isb, own, nbr)]
    bf = np.flatnonzero(isb)
    if len(bf):
        # _precompute_ghost_states (inviscid_p0.py:112-143) stores the ghost
        # state per owner CELL, overwritten face by face in record order: every
        # boundary face of a cell uses the ghost state of that cell's last
        # boundary face
        G = ghost_states(m, Q[:, None, :], bf)[1][:, 0, :]
        Gcell = np.zeros((N, 5))
        Gcell[own[bf]] = G  # later faces overwrite earlier ones (numpy assigns in index order)
        Qn[bf] = Gcell[own[bf]]
    F = ausm_up(Q[own], Qn, n) * area[:, None]
    R = np.zeros((N, 5))
    for f in range(len(own)):
        R[own[f]] -= F[f] * (1.0 / vol[own[f]])
        if not isb[f]:
            R[nbr[f]] += F[f] * (1.0 / vol[nbr[f]])
    return R[:, None, :]


def inviscid_residual(m: Mesh, U):
    """compute_inviscid_residual_fr, core/fr_residual/inviscid.py:139-345,
    with the colored interface kernel core/fr_residual/inviscid_kernel_colored.py:43-236
    (order 0: the finite-volume path, inviscid.py:164-170)."""
    if m.S == 1:
        return inviscid_residual_p0(m, U)
    N, S = m.N, m.S
    Q = conserved_to_primitive(U[..., :5])
    det = m.c["det_jacs"]
    adj = m.extras["adj"]
    Fn = int(m.c["n_fine"])
    div_fine = np.zeros((N, Fn, 5))
    Qf = np.zeros((N, Fn, 5))
    for sl, t in m.split():
        Qf[sl] = contract_1axis(m.c["c2f_" + t], Q[sl])
    Ft = np.matmul(m.extras["adj_fine"], euler_flux(Qf))
    for sl, t in m.split():
        div_fine[sl] = contract_2axis(m.c["Dfine_" + t], Ft[sl])
    div = np.zeros((N, S, 5))
    for sl, t in m.split():
        div[sl] = contract_1axis(m.c["f2c_" + t], div_fine[sl])
    R = -div / det[..., None]

    corr = np.zeros((N, S, 5))
    isb = m.c["is_boundary"].astype(bool)
    opr = m.c["owner_is_primary"].astype(bool)
    npr = m.c["neighbor_is_primary"].astype(bool)
    bfaces = np.flatnonzero(isb & opr)
    Qghost = np.zeros(m.c["true_normal"].shape[:2] + (5,))
    if len(bfaces):
        Qghost[bfaces] = ghost_states(m, Q, bfaces)[1]
    for faces in _color_faces(m):
        # owner side
        f = faces[opr[faces]]
        if len(f):
            _inviscid_side(m, Q, adj, det, f, owner=True, Qghost=Qghost, isb=isb, corr=corr)
        f = faces[(~isb[faces]) & npr[faces]]
        if len(f):
            _inviscid_side(m, Q, adj, det, f, owner=False, Qghost=Qghost, isb=isb, corr=corr)
    R = R + corr
    return suppress_outliers(R, U[..., :5])


def _side_geometry(m: Mesh, f, owner):
    if owner:
        cell, ax, sd = m.c["owner_cell"][f], m.c["owner_axis"][f], m.c["owner_side"][f]
    else:
        cell, ax, sd = m.c["neighbor_cell"][f], m.c["neighbor_axis"][f], m.c["neighbor_side"][f]
    return cell, ax, sd


def _inviscid_side(m, Q, adj, det, f, owner, Qghost, isb, corr):
    cell, ax, sd = _side_geometry(m, f, owner)
    E = extrap_E(m, cell, ax, sd)
    Qs = np.matmul(E, Q[cell])  # (F,P,5)
    arow = np.matmul(E, adj[cell, :, ax, :])  # (F,P,3)
    a0, a1, a2 = arow[..., 0], arow[..., 1], arow[..., 2]
    mag = np.sqrt(a0 * a0 + a1 * a1 + a2 * a2)
    mag = np.where(mag < 1e-300, 1e-300, mag)
    s = sd[:, None]
    d = np.stack([a0 / mag * s, a1 / mag * s, a2 / mag * s], axis=-1)
    tn = m.c["true_normal"][f] if owner else -m.c["true_normal"][f]
    align = d[..., 0] * tn[..., 0] + d[..., 1] * tn[..., 1] + d[..., 2] * tn[..., 2]
    d = np.where((align < 0.5)[..., None], tn, d)
    if owner:
        Qn = gather_sources(m, f, Q, "nb")
        bnd = isb[f]
        Qn[bnd] = Qghost[f[bnd]]
        Fc = ausm_up(Qs, Qn, d)
    else:
        Qo = gather_sources(m, f, Q, "ow")
        Fc = ausm_up(Qs, Qo, d)
    Fcom = Fc * (mag * s)[..., None]
    Fp = euler_flux(Qs)
    Fown = a0[..., None] * Fp[..., 0, :] + a1[..., None] * Fp[..., 1, :] + a2[..., None] * Fp[..., 2, :]
    jump = Fcom - Fown
    contrib = distribute(m, jump, ax, sd)
    corr[cell] += -contrib / det[cell][..., None]


def viscous_residual(m: Mesh, U, mu, mu_t):
    """compute_viscous_residual_fr, core/fr_residual/viscous_flux.py:113-302,
    colored interface kernel core/fr_residual/viscous_flux_kernel.py:292-520."""
    N, S = m.N, m.S
    mu_t = np.zeros((N, S)) if mu_t is None else mu_t
    Q = conserved_to_primitive(U[..., :5])
    T = Q[..., 4] / (np.maximum(Q[..., 0], 1e-10) * R_AIR)
    gQ = physical_gradient(m, Q)
    gv = gQ[:, :, 1:4, :]
    gT = physical_gradient(m, T[:, :, None])[:, :, 0, :]
    det = m.c["det_jacs"]
    adj = m.extras["adj"]
    G = viscous_flux(Q, gv, gT, mu, mu_t)
    Gt = np.matmul(adj, G)
    div = np.zeros((N, S, 5))
    for sl, t in m.split():
        div[sl] = contract_2axis(m.c["D_3d_" + t], Gt[sl])
    R = div / det[..., None]

    corr = np.zeros((N, S, 5))
    isb = m.c["is_boundary"].astype(bool)
    opr = m.c["owner_is_primary"].astype(bool)
    npr = m.c["neighbor_is_primary"].astype(bool)
    bfaces = np.flatnonzero(isb & opr)
    Qghost = np.zeros(m.c["true_normal"].shape[:2] + (5,))
    if len(bfaces):
        Qghost[bfaces] = ghost_states(m, Q, bfaces)[1]
    gflat = np.concatenate([gv.reshape(N, S, 9), gT, mu_t[..., None]], axis=-1)  # (N,S,13)
    for faces in _color_faces(m):
        f = faces[opr[faces]]
        if len(f):
            _viscous_side(m, Q, gflat, adj, det, mu, f, True, Qghost, isb, corr)
        f = faces[(~isb[faces]) & npr[faces]]
        if len(f):
            _viscous_side(m, Q, gflat, adj, det, mu, f, False, Qghost, isb, corr)
    R = R + corr
    return suppress_outliers(R, U[..., :5])


def _viscous_side(m, Q, gflat, adj, det, mu, f, owner, Qghost, isb, corr):
    cell, ax, sd = _side_geometry(m, f, owner)
    E = extrap_E(m, cell, ax, sd)
    Qs = np.matmul(E, Q[cell])
    gs = np.matmul(E, gflat[cell])  # (F,P,13)
    arow = np.matmul(E, adj[cell, :, ax, :])
    if owner:
        Qn = gather_sources(m, f, Q, "nb")
        gn = gather_sources(m, f, gflat, "nb")
        bnd = isb[f]
        Qn[bnd] = Qghost[f[bnd]]
        gn[bnd] = gs[bnd]
    else:
        Qn = gather_sources(m, f, Q, "ow")
        gn = gather_sources(m, f, gflat, "ow")
    Qa = 0.5 * (Qs + Qn)
    ga = 0.5 * (gs + gn)
    Gc = viscous_flux(Qa, ga[..., :9].reshape(ga.shape[:2] + (3, 3)), ga[..., 9:12], mu, ga[..., 12])
    Go = viscous_flux(Qs, gs[..., :9].reshape(gs.shape[:2] + (3, 3)), gs[..., 9:12], mu, gs[..., 12])
    a0, a1, a2 = arow[..., 0:1], arow[..., 1:2], arow[..., 2:3]
    Gtc = a0 * Gc[..., 0, :] + a1 * Gc[..., 1, :] + a2 * Gc[..., 2, :]
    Gto = a0 * Go[..., 0, :] + a1 * Go[..., 1, :] + a2 * Go[..., 2, :]
    jump = Gtc - Gto
    if owner:
        bnd = isb[f]
        if np.any(bnd):
            # viscous_boundary_penalty_tilde, core/fr_operators/flux_kernels.py:140-200
            vol = np.sum(det[cell[bnd]], axis=1) / m.S  # viscous_flux_kernel.py:344-347
            h = vol ** (1.0 / 3.0)
            h = np.where(h < 1e-300, 1e-300, h)
            mag = np.sqrt(arow[bnd, :, 0] * arow[bnd, :, 0] + arow[bnd, :, 1] * arow[bnd, :, 1]
                          + arow[bnd, :, 2] * arow[bnd, :, 2])
            eta = C_IP * (mu + gs[bnd, :, 12]) / h[:, None]
            scale = eta * mag * sd[bnd][:, None]
            pen = -scale[..., None] * (Qs[bnd, :, 1:4] - Qn[bnd, :, 1:4])
            jb = jump[bnd]
            jb[..., 1:4] = jb[..., 1:4] + pen
            jump[bnd] = jb
    contrib = distribute(m, jump, ax, sd)
    corr[cell] += contrib / det[cell][..., None]


# ---------------------------------------------------------------------------
# local time step, filter, positivity
# ---------------------------------------------------------------------------
def local_dt(m: Mesh, Q, mu, mu_t):
    """compute_local_time_step, core/fr_solver/cfl.py:12-147 with
    _get_metric_flux_scale, core/fr_solver/solver_geometry.py:18-32."""
    rho, u, v, w, p = (Q[..., i] for i in range(5))
    a = np.sqrt(np.maximum(1.4 * p / np.maximum(rho, 1e-10), 1e-10))
    vm = np.sqrt(u**2 + v**2 + w**2)
    wave = np.maximum(vm + a, 1e-10)
    h = np.power(np.abs(m.c["cell_volumes"]), 1.0 / 3.0)
    hx = np.tile(h[:, None], (1, m.S))
    CFL = 0.1
    P = m.order
    fa = 1.0 / (2 * P + 1)
    fv = 1.0 / (2 * P + 1) ** 2
    dt_adv = CFL * fa * hx / wave
    mu_eff = mu + mu_t if mu_t is not None else np.full_like(rho, mu)
    dt_visc = 0.25 * CFL * fv * rho * hx**2 / np.maximum(mu_eff, 1e-30)
    mfs = metric_flux_scale(m) if "mfs" not in m.extras else m.extras["mfs"]
    dt_geo = CFL * np.abs(m.c["det_jacs"]) / np.maximum(mfs * wave, 1e-300)
    return np.minimum(np.minimum(dt_adv, dt_visc), dt_geo)


def metric_flux_scale(m: Mesh):
    """_get_metric_flux_scale, core/fr_solver/solver_geometry.py:18-32: sum_m |adj(J)[m,:]|."""
    return np.sum(np.linalg.norm(m.extras["adj"], axis=-1), axis=-1)


def modal_filter(m: Mesh, U):
    """_filter_flat_U, core/fr_solver/filter.py:29-42 (first 5 variables)."""
    U = U.copy()
    for sl, t in m.split():
        U[sl, :, :5] = np.einsum("sj,cjv->csv", m.c["filter_" + t], U[sl, :, :5])
    return U


def enforce_positivity(Uf, p_floor=1.0):
    """core/time_integration/positivity.py:13-45 on the flat (N*S, n_vars) array, in place."""
    rho = np.maximum(Uf[:, 0], 1e-6)
    Uf[:, 0] = rho
    vel = Uf[:, 1:4] / rho[:, None]
    vm = np.sqrt(np.sum(vel**2, axis=1))
    clip = vm > 1e4
    if np.any(clip):
        vel[clip] *= (1e4 / vm[clip])[:, None]
        Uf[clip, 1:4] = rho[clip, None] * vel[clip]
    ke = 0.5 * rho * np.sum(vel**2, axis=1)
    p = (GAMMA - 1.0) * (Uf[:, 4] - ke)
    low = p < p_floor
    if np.any(low):
        Uf[low, 4] = p_floor / (GAMMA - 1.0) + ke[low]
    if Uf.shape[1] > 5:
        Uf[:, 5] = np.maximum(Uf[:, 5], 0.0)
    if Uf.shape[1] > 6:
        Uf[:, 6] = np.maximum(Uf[:, 6], 1e-8)
    return Uf


# ---------------------------------------------------------------------------
# SST k-omega
# ---------------------------------------------------------------------------
def _F1(k, w, d, nu, rho, CD):
    """compute_blending_function_F1, core/turbulence/sst.py:92-141."""
    w = np.maximum(w, 1e-10)
    k = np.maximum(k, 1e-10)
    d = np.maximum(d, 1e-10)
    sk = np.sqrt(k)
    t1 = sk / (SST["beta_star"] * w * d)
    t2 = 500.0 * nu / (d**2 * w)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        t3 = 4.0 * rho * SST["sigma_w2"] * k / (np.maximum(CD, 1e-10) * d**2)
    a = np.minimum(np.maximum(t1, t2), t3)
    a = np.where(np.isfinite(a), a, 1e75)
    a = np.minimum(a, 1e75)
    with np.errstate(over="ignore"):
        return np.tanh(a**4)


def _F2(k, w, d, nu):
    """compute_blending_function_F2, core/turbulence/sst.py:143-179."""
    w = np.maximum(w, 1e-10)
    k = np.maximum(k, 1e-10)
    d = np.maximum(d, 1e-10)
    sk = np.sqrt(k)
    a = np.maximum(2.0 * sk / (SST["beta_star"] * w * d), 500.0 * nu / (d**2 * w))
    a = np.where(np.isfinite(a), a, 1e150)
    a = np.minimum(a, 1e150)
    with np.errstate(over="ignore"):
        return np.tanh(a**2)


def strain_mag(g):
    """compute_strain_rate_magnitude, core/turbulence/sst.py:74-90."""
    Sij = 0.5 * (g + np.transpose(g, (0, 1, 3, 2)))
    return np.sqrt(2.0 * np.einsum("nijm,nijm->ni", Sij, Sij))


def _clip_grad(g):
    """|grad| <= 1e6 clip, core/fr_solver/turbulence.py:244-255 (same as transport.py:448-457)."""
    with np.errstate(over="ignore", invalid="ignore"):
        mag = np.linalg.norm(g, axis=-1)
        if np.any(mag > 1e6):
            sc = 1e6 / np.maximum(mag, 1e-10)
            g = g * np.clip(sc, 0, 1)[..., None]
    return g


def _extrap_scalar(m: Mesh, phi, wall_zero=None):
    """extrapolate_scalar_to_faces_kernel, core/turbulence/transport_kernel.py:25-173."""
    oc = m.c["owner_cell"]
    side = m.c["owner_side"]
    ct = (oc >= m.n_prism).astype(np.int64)
    si = np.where(side <= 0.0, 0, 1)
    E = m.c["boundary_extrap"][ct, m.c["owner_axis"], si]
    po = np.einsum("fps,fs->fp", E, phi[oc])
    allf = np.arange(len(oc))
    pn = gather_sources(m, allf, phi[..., None], "nb")[..., 0]
    nosrc = (m.c["nb_src0_cell"] < 0) & (m.c["nb_src1_idx"] < 0)
    wz = np.zeros(len(oc), bool) if wall_zero is None else wall_zero
    pn = np.where((nosrc & wz)[:, None], -po, np.where(nosrc[:, None], po, pn))
    return po, pn


def _distribute_scalar(m: Mesh, corr_fp):
    """distribute_corrections_to_cells_kernel_colored, core/turbulence/transport_kernel.py:269-327
    (every face, owner side subtracts, neighbour side adds, in color order)."""
    det = m.c["det_jacs"]
    out = np.zeros((m.N, m.S))
    oc, nc = m.c["owner_cell"], m.c["neighbor_cell"]
    for faces in _color_faces(m):
        o = oc[faces]
        ax, sd = m.c["owner_axis"][faces], m.c["owner_side"][faces]
        fp = m.c["dist_fp_of_sp"][ax]
        co = m.c["dist_axis_coord_of_sp"][ax]
        g = np.where((sd > 0)[:, None], m.c["g_right"][co], m.c["g_left"][co])
        contrib = g * np.take_along_axis(corr_fp[faces], fp, axis=1)
        out[o] -= contrib / det[o]
        inner = nc[faces] >= 0
        fi = faces[inner]
        if len(fi):
            n = nc[fi]
            ax, sd = m.c["neighbor_axis"][fi], m.c["neighbor_side"][fi]
            fp = m.c["dist_fp_of_sp"][ax]
            co = m.c["dist_axis_coord_of_sp"][ax]
            g = np.where((sd > 0)[:, None], m.c["g_right"][co], m.c["g_left"][co])
            contrib = g * np.take_along_axis(corr_fp[fi], fp, axis=1)
            out[n] += contrib / det[n]
    return out


def _div_scalar_flux(m: Mesh, Fphys):
    """sum_m tensordot(F~[:,:,m], D[:,:,m]), core/turbulence/transport.py:157-171."""
    Ft = np.matmul(m.extras["adj"], Fphys[..., None])[..., 0]
    div = np.zeros((m.N, m.S))
    for sl, t in m.split():
        D = m.c["D_3d_" + t]
        for k in range(3):
            div[sl] += np.tensordot(Ft[sl, :, k], D[:, :, k], axes=([1], [1]))
    return div


def scalar_convection(m: Mesh, phi, rho, vel, wall_zero=None):
    """compute_scalar_convection_residual, core/turbulence/transport.py:122-222."""
    with np.errstate(over="ignore", invalid="ignore"):
        R = -_div_scalar_flux(m, rho[..., None] * vel * phi[..., None]) / m.c["det_jacs"]
    ro, _ = _extrap_scalar(m, rho)
    vo = np.stack([_extrap_scalar(m, vel[:, :, d])[0] for d in range(3)], axis=-1)
    po, pn = _extrap_scalar(m, phi, wall_zero)
    mflux = np.sum((ro[..., None] * vo) * m.c["true_normal"], axis=-1)
    up = np.where(mflux >= 0, po, pn)
    corr = _distribute_scalar(m, mflux * (up - po))
    with np.errstate(over="ignore", invalid="ignore"):
        return R + corr


def scalar_diffusion(m: Mesh, phi, gamma, wall_zero=None):
    """compute_scalar_diffusion_residual, core/turbulence/transport.py:225-332."""
    g = physical_gradient(m, phi[..., None])[:, :, 0, :]
    with np.errstate(over="ignore", invalid="ignore"):
        R = -_div_scalar_flux(m, gamma[..., None] * g) / m.c["det_jacs"]
    po, pn = _extrap_scalar(m, phi, wall_zero)
    go, gn = _extrap_scalar(m, gamma)
    with np.errstate(over="ignore", invalid="ignore"):
        corr = _distribute_scalar(m, (0.5 * (go + gn)) * (0.5 * (po + pn) - po))
        return R - corr


def wall_face_mask(m: Mesh):
    """_compute_wall_dirichlet_face_mask, core/turbulence/transport.py:335-364."""
    return m.c["bc_type"][m.c["bc_group"]] == BC_WALL


@dataclass
class TurbState:
    k: np.ndarray
    w: np.ndarray
    nut: np.ndarray
    beta_blend: Optional[np.ndarray] = None


def sst_source_and_update(m: Mesh, U, Q, turb: TurbState, dt, mu_mol, wall_distance):
    """compute_turbulence_source, core/fr_solver/turbulence.py:178-330, with
    SSTModelFR.compute_source_terms / update_fields (core/turbulence/sst.py:241-479) and
    compute_turbulence_transport_residual (core/turbulence/transport.py:367-522).
    Updates ``turb`` in place and returns (Sk, Sw, transport_k, transport_w)."""
    gU = physical_gradient(m, U)
    gvel = gU[:, :, 1:4, :]
    gk = _clip_grad(physical_gradient(m, turb.k[..., None])[:, :, 0, :])
    gw = _clip_grad(physical_gradient(m, turb.w[..., None])[:, :, 0, :])
    rho = Q[:, :, 0]
    # --- compute_source_terms (mu = 1.8e-5 hard-coded) ---
    nu = MU_SST_SOURCE / np.maximum(rho, 1e-10)
    k_s = np.minimum(turb.k, 1e40)
    w_s = np.maximum(np.minimum(turb.w, 1e40), 1e-10)
    Sm = strain_mag(gvel)
    gd = np.sum(gk * gw, axis=2)
    CD = np.maximum(2.0 * rho * SST["sigma_w2"] / w_s * gd, 1e-10)
    F1 = _F1(k_s, w_s, wall_distance, nu, rho, CD)
    F2 = _F2(k_s, w_s, wall_distance, nu)
    beta = F1 * SST["beta1"] + (1.0 - F1) * SST["beta2"]
    kk = np.maximum(k_s, 1e-10)
    ww = np.maximum(w_s, 1e-10)
    SS = np.maximum(Sm, 1e-10)
    with np.errstate(over="ignore", invalid="ignore"):
        nut = SST["a1"] * kk / np.maximum(SST["a1"] * ww, F2 * SS)
    nut = np.minimum(nut, SST["tvr_max"] * MU_SST_SOURCE / np.maximum(rho, 1e-10))
    nut = np.where(np.isfinite(nut), nut, 0.0)
    Pk = nut * rho * Sm**2
    Pk = np.minimum(Pk, 10.0 * SST["beta_star"] * rho * k_s * w_s)
    Dk = rho * SST["beta_star"] * k_s * w_s
    Sk = Pk - Dk
    bs = SST["beta_star"]
    g1 = SST["beta1"] / bs - SST["sigma_w1"] * SST["kappa"] ** 2 / np.sqrt(bs)
    g2 = SST["beta2"] / bs - SST["sigma_w2"] * SST["kappa"] ** 2 / np.sqrt(bs)
    gam = F1 * g1 + (1.0 - F1) * g2
    Sw = rho * gam * Sm**2 - rho * beta * w_s**2 + 2.0 * rho * (1.0 - F1) * SST["sigma_w2"] / w_s * gd
    Sk = np.where(np.isfinite(Sk), Sk, 0.0)
    Sw = np.where(np.isfinite(Sw), Sw, 0.0)
    turb.nut = nut
    turb.beta_blend = beta
    # --- transport (mu = solver.mu_molecular) ---
    vel = Q[:, :, 1:4]
    rnut = rho * turb.nut
    nu_m = mu_mol / np.maximum(rho, 1e-10)
    with np.errstate(over="ignore", invalid="ignore"):
        gd2 = np.sum(gk * gw, axis=-1)
        CD2 = np.maximum(2.0 * rho * SST["sigma_w2"] / np.maximum(turb.w, 1e-10) * gd2, 1e-10)
    F1t = _F1(turb.k, turb.w, wall_distance, nu_m, rho, CD2)
    sk_ = F1t * SST["sigma_k1"] + (1.0 - F1t) * SST["sigma_k2"]
    sw_ = F1t * SST["sigma_w1"] + (1.0 - F1t) * SST["sigma_w2"]
    gk_ = mu_mol + sk_ * rnut
    gw_ = mu_mol + sw_ * rnut
    wall = wall_face_mask(m)
    with np.errstate(over="ignore", invalid="ignore"):
        tk = (scalar_convection(m, turb.k, rho, vel, wall) + scalar_diffusion(m, turb.k, gk_, wall)) / \
            np.maximum(rho, 1e-10)
        tw = (scalar_convection(m, turb.w, rho, vel) + scalar_diffusion(m, turb.w, gw_)) / np.maximum(rho, 1e-10)
    tk = suppress_outliers(tk[:, :, None], turb.k[:, :, None])[:, :, 0]
    tw = suppress_outliers(tw[:, :, None], turb.w[:, :, None])[:, :, 0]
    tk = np.where(np.isfinite(tk), tk, 0.0)
    tw = np.where(np.isfinite(tw), tw, 0.0)
    # --- update_fields ---
    dk = Sk / np.maximum(rho, 1e-10)
    dw = Sw / np.maximum(rho, 1e-10)
    wo = np.maximum(turb.w, 1e-10)
    with np.errstate(over="ignore", invalid="ignore"):
        dkd = dk / (1.0 + dt * (SST["beta_star"] * wo))
        dwd = dw / (1.0 + dt * (beta * wo))
    dkd = np.where(np.isfinite(dkd), dkd, 0.0)
    dwd = np.where(np.isfinite(dwd), dwd, 0.0)
    kt = dkd + tk
    wt = dwd + tw
    kt = np.where(np.isfinite(kt), kt, 0.0)
    wt = np.where(np.isfinite(wt), wt, 0.0)
    k_new = turb.k + dt * kt
    w_new = turb.w + dt * wt
    k_new = np.where(np.isfinite(k_new), k_new, 1e-12)
    w_new = np.where(np.isfinite(w_new), w_new, 1e-12)
    turb.k = np.maximum(k_new, 1e-12)
    turb.w = np.maximum(w_new, 1e-12)
    return Sk, Sw, tk, tw


# ---------------------------------------------------------------------------
# the step
# ---------------------------------------------------------------------------
@dataclass
class Solver:
    """State of one case: conserved U (N,S,n_vars), turbulence fields, settings."""

    m: Mesh
    U: np.ndarray
    mu: float
    turb: Optional[TurbState] = None
    wall_distance: Optional[np.ndarray] = None
    inviscid_only: bool = False
    global_dt_factor: float = 0.0
    time_scheme: str = "ssp_rk3"
    dt_step: float = 1e-3            # physical step of the dual-time scheme
    dual_time_inner_iter: int = 20
    U_prev: Optional[np.ndarray] = None  # dual time: state at the previous physical level

    def mu_t(self, Q):
        """get_turbulent_viscosity_field, core/fr_solver/turbulence.py:355-366."""
        if self.turb is None:
            return None
        return Q[:, :, 0] * self.turb.nut

    def residual(self, U):
        """-(inviscid + viscous), the mean_flow_residual closure of core/fr_solver/step.py:121-132."""
        Q = state_primitives(U)
        Ri = inviscid_residual(self.m, U)
        full = np.zeros_like(U)
        full[:, :, :5] = Ri
        if not self.inviscid_only:
            full[:, :, :5] += viscous_residual(self.m, U, self.mu, self.mu_t(Q))
        return -full

    def _parts(self, U):
        """(inviscid, viscous) residuals dU/dt of U, zero turbulence columns."""
        Q = state_primitives(U)
        Ri = np.zeros_like(U)
        Rv = np.zeros_like(U)
        Ri[:, :, :5] = inviscid_residual(self.m, U)
        if not self.inviscid_only:
            Rv[:, :, :5] = viscous_residual(self.m, U, self.mu, self.mu_t(Q))
        return Ri, Rv

    def _ssp_rk3(self, U0, rfun, dtc, residual0):
        """TimeIntegrator._ssp_rk_stage_step with the RK3 table and the filter,
        core/time_integration/base.py:250-335; rfun(U) -> R (dU/dt = -R)."""
        m = self.m
        N, S, nv = self.U.shape
        L0 = -residual0
        U1 = U0 + dtc * L0
        enforce_positivity(U1)
        U1 = modal_filter(m, U1.reshape(N, S, nv)).reshape(N * S, nv)
        L1 = -rfun(U1)
        U2 = 0.75 * U0 + 0.25 * U1 + 0.25 * dtc * L1
        enforce_positivity(U2)
        U2 = modal_filter(m, U2.reshape(N, S, nv)).reshape(N * S, nv)
        L2 = -rfun(U2)
        U3 = 1.0 / 3.0 * U0 + 0.0 * U1 + 2.0 / 3.0 * U2 + 2.0 / 3.0 * dtc * L2
        enforce_positivity(U3)
        return modal_filter(m, U3.reshape(N, S, nv)).reshape(N * S, nv)

    def _dual_time(self, U_flat, dt_local, dt_phys):
        """step_dual_time, core/time_integration/dual.py:19-158."""
        N, S, nv = self.U.shape
        U_n = U_flat
        U_tau = U_n.copy()
        prev = self.U_prev

        def spatial(Uf):
            return self.residual(Uf.reshape(N, S, nv)).reshape(N * S, nv)

        if prev is None:
            def dual(Uf):
                return spatial(Uf) + (Uf - U_n) / dt_phys
        else:
            def dual(Uf):
                return spatial(Uf) + (3.0 * Uf - 4.0 * U_n + prev) / (2.0 * dt_phys)

        init = np.linalg.norm(dual(U_tau))
        cfl = 0.1
        prev_norm = None
        for k in range(self.dual_time_inner_iter):
            R = dual(U_tau)
            cur = np.linalg.norm(R)
            if cur < init * 1e-6:
                break
            if k >= 1 and cur < 1e-4:
                break
            if k > 0:
                ratio = cur / prev_norm
                if ratio < 0.5:
                    cfl = min(cfl * 1.5, 10.0)
                elif ratio > 1.0:
                    cfl = max(cfl * 0.5, 0.1)
            prev_norm = cur
            dtc = (dt_local * cfl)[:, None]
            U_next = self._ssp_rk3(U_tau, dual, dtc, R)
            enforce_positivity(U_next)
            U_next = modal_filter(self.m, U_next.reshape(N, S, nv)).reshape(N * S, nv)
            if np.linalg.norm(U_next - U_tau) < 1e-10:
                break
            U_tau = U_next
        return U_tau

    def _imex(self, U_flat, dt_local):
        """step_imex, core/time_integration/imex.py:17-97."""
        N, S, nv = self.U.shape
        Ri, _ = self._parts(U_flat.reshape(N, S, nv))
        R_exp = -Ri.reshape(N * S, nv)

        def r_imp(Uf):
            return -self._parts(Uf.reshape(N, S, nv))[1].reshape(N * S, nv)

        U_new = U_flat.copy()
        dt_vec = dt_local[:, None]
        init = np.linalg.norm(R_exp + r_imp(U_flat))
        damping, prev_norm = 0.5, None
        for it in range(5):
            total = R_exp + r_imp(U_new)
            cur = np.linalg.norm(total)
            if it > 0:
                ratio = cur / prev_norm
                if ratio < 0.5:
                    damping = min(damping * 1.2, 1.0)
                elif ratio > 1.0:
                    damping = max(damping * 0.5, 0.1)
            else:
                damping = 0.5
            prev_norm = cur
            U_next = U_new - dt_vec * total * damping
            enforce_positivity(U_next)
            if np.linalg.norm(U_next - U_new) < 1e-8 or cur < init * 1e-6:
                break
            U_new = U_next
        return U_new

    def step(self):
        """FRSolver.step, core/fr_solver/step.py:15-221 (SSP-RK3, DUAL_TIME and
        IMEX_EULER branches)."""
        if self.time_scheme != "ssp_rk3":
            return self._step_scheme()
        m = self.m
        N, S, nv = self.U.shape
        Q = state_primitives(self.U)
        dt = local_dt(m, Q, self.mu, self.mu_t(Q))
        if self.global_dt_factor:
            dt = np.full((N, S), self.global_dt_factor * float(np.min(dt)))
        if self.turb is not None:
            sst_source_and_update(m, self.U, Q, self.turb, dt, self.mu, self.wall_distance)
        U0 = self.U.reshape(N * S, nv).copy()
        dtc = dt.reshape(N * S)[:, None]
        R0 = self.residual(self.U).reshape(N * S, nv)
        dUdt = -R0
        # TimeIntegrator._ssp_rk_stage_step, core/time_integration/base.py:250-335
        L0 = -R0
        U1 = U0 + dtc * L0
        enforce_positivity(U1)
        U1 = modal_filter(m, U1.reshape(N, S, nv)).reshape(N * S, nv)
        L1 = -self.residual(U1.reshape(N, S, nv)).reshape(N * S, nv)
        U2 = 0.75 * U0 + 0.25 * U1 + 0.25 * dtc * L1
        enforce_positivity(U2)
        U2 = modal_filter(m, U2.reshape(N, S, nv)).reshape(N * S, nv)
        L2 = -self.residual(U2.reshape(N, S, nv)).reshape(N * S, nv)
        U3 = 1.0 / 3.0 * U0 + 0.0 * U1 + 2.0 / 3.0 * U2 + 2.0 / 3.0 * dtc * L2
        enforce_positivity(U3)
        U3 = modal_filter(m, U3.reshape(N, S, nv)).reshape(N * S, nv)
        self.U = U3.reshape(N, S, nv)
        return float(np.linalg.norm(dUdt) / np.sqrt(dUdt.size))

    def _step_scheme(self):
        m = self.m
        N, S, nv = self.U.shape
        Q = state_primitives(self.U)
        dt = local_dt(m, Q, self.mu, self.mu_t(Q))
        if self.global_dt_factor:
            dt = np.full((N, S), self.global_dt_factor * float(np.min(dt)))
        if self.turb is not None:
            turb_dt = np.full((N, S), self.dt_step) if self.time_scheme == "dual_time" else dt
            sst_source_and_update(m, self.U, Q, self.turb, turb_dt, self.mu, self.wall_distance)
        U_flat = self.U.reshape(N * S, nv).copy()
        dUdt = -self.residual(self.U).reshape(N * S, nv)
        if self.time_scheme == "dual_time":
            U_new = self._dual_time(U_flat, dt.reshape(N * S), self.dt_step)
            self.U_prev = U_flat.copy()
        else:
            U_new = self._imex(U_flat, dt.reshape(N * S))
        self.U = U_new.reshape(N, S, nv)
        return float(np.linalg.norm(dUdt) / np.sqrt(dUdt.size))


def cd_cl(m: Mesh, U, mu, nut, freestream, reference_area=1.0):
    """compute_aerodynamic_coefficients_fr, postprocess/fr_coefficients.py:27-152 -> (Cd, Cl, Cs)."""
    Q = state_primitives(U)
    mu_t = None if nut is None else Q[:, :, 0] * nut
    faces = np.flatnonzero(m.c["cd_wall_face"].astype(bool) & m.c["owner_is_primary"].astype(bool))
    gQ = physical_gradient(m, Q)
    gv = gQ[:, :, 1:4, :]
    oc = m.c["owner_cell"][faces]
    E = extrap_E(m, oc, m.c["owner_axis"][faces], m.c["owner_side"][faces])
    Qf = np.matmul(E, Q[oc])
    n = m.c["true_normal"][faces]
    aw = m.c["true_area_weight"][faces]
    Fp = np.zeros(3)
    Fv = np.zeros(3)
    for i in range(len(faces)):
        Fp += np.sum(Qf[i, :, 4][:, None] * n[i] * aw[i][:, None], axis=0)
        g = (E[i] @ gv[oc[i]].reshape(m.S, 9)).reshape(-1, 3, 3)
        mt = E[i] @ mu_t[oc[i]][:, None] if mu_t is not None else np.zeros((g.shape[0], 1))
        mtot = mu + mt[:, 0]
        Sij = 0.5 * (g + np.swapaxes(g, -1, -2))
        div = g[:, 0, 0] + g[:, 1, 1] + g[:, 2, 2]
        tau = 2.0 * mtot[:, None, None] * Sij + (-2.0 / 3.0 * mtot)[:, None, None] * div[:, None, None] * np.eye(3)
        tr = np.einsum("fij,fj->fi", tau, n[i])
        Fv += -np.sum(tr * aw[i][:, None], axis=0)
    F = Fp + Fv
    rho_inf, vel_inf = freestream[0], freestream[1]
    q = 0.5 * rho_inf * vel_inf**2
    den = max(q * reference_area, 1e-300)
    return np.array([F[0] / den, F[2] / den, F[1] / den])


# ---------------------------------------------------------------------------
# order continuation
# ---------------------------------------------------------------------------
def interp_matrix_3d(old_1d, new_1d):
    """_build_linear_interp_matrix_3d, core/utils/order_continuation.py:14-60:
    column k is scipy's RegularGridInterpolator(method="linear",
    fill_value=None) of the k-th unit vector on the old tensor grid, at the
    new grid's points (meshgrid "ij", first coordinate slowest)."""
    from scipy.interpolate import RegularGridInterpolator

    n_old, n_new = len(old_1d), len(new_1d)
    X, Y, Z = np.meshgrid(new_1d, new_1d, new_1d, indexing="ij")
    pts = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    W = np.zeros((n_new**3, n_old**3))
    for k in range(n_old**3):
        e = np.zeros(n_old**3)
        e[k] = 1.0
        f = RegularGridInterpolator((old_1d, old_1d, old_1d), e.reshape(n_old, n_old, n_old), method="linear",
                                    bounds_error=False, fill_value=None)
        W[:, k] = f(pts)
    return W


def order_continuation(case_for_order, order, mu, inviscid_only, freestream, max_iter, dt, tol, turb=None,
                       wall_distance=None):
    """run_order_continuation, core/utils/order_continuation.py:207-425, on
    the oracle's solver: restart from the uniform free stream at P0
    (FRState.initialize_uniform, core/fr_solver/state.py:50-74), phases
    P0..order of max_iter // (order + 1) steps, phase tolerance
    tol * 10**(order - p), an early move on after >= 20 steps once the
    residual dropped 100x, the state prolonged between phases by
    np.einsum("ab,cbv->cav", W, U) (interpolate_to_new_order, :62-124).

    With ``turb == "SST"`` (core/utils/order_continuation.py:120-144, 245-276):
    the restart sets k = 1e-6, omega = 1, nu_t = 0 and the wall distance to
    the cell means of ``wall_distance`` (the target order's field); k, omega,
    nu_t and the wall distance are prolonged by np.einsum("ab,cb->ca", W, .)
    between phases.

    Returns (step_order, step_residual, states, result): ``states`` maps
    "U_start_p<p>" / "U_end_p<p>" to the phase's first and last states (and
    "k_end_p<p>", "w_end_p<p>", "nut_end_p<p>" with SST)."""
    rho, u, p = freestream
    c0 = case_for_order(0)
    N = int(c0["n_cells"])
    e = p / ((GAMMA - 1.0) * rho) + 0.5 * (u**2 + 0.0**2 + 0.0**2)
    sst = turb == "SST"
    U = np.zeros((N, 1, 7 if sst else 5))
    U[:, :, 0], U[:, :, 1], U[:, :, 2], U[:, :, 3], U[:, :, 4] = rho, rho * u, rho * 0.0, rho * 0.0, rho * e
    tk = tw = tn = wd = None
    if sst:
        # FRState.initialize_uniform's turbulence columns (k 1e-6, omega 1e-2)
        U[:, :, 5], U[:, :, 6] = rho * 1e-6, rho * 1e-2
        tk, tw, tn = np.full((N, 1), 1e-6), np.ones((N, 1)), np.zeros((N, 1))
        wd = np.tile(np.mean(wall_distance, axis=1, keepdims=True), (1, 1))
    orders = list(range(0, order + 1))
    step_order, step_res, states = [], [], {}
    total, final = 0, 1e10
    cur = 0
    # the solver caches the metric flux scale at its first local time step
    # (the P0 phase) and reuses it, broadcast over the points, while the cell
    # count is unchanged (solver_geometry.py:18-32, cfl.py:136-146)
    mfs_cache = None
    for tp in orders:
        if tp > 0:
            W = interp_matrix_3d(np.polynomial.legendre.leggauss(cur + 1)[0], np.polynomial.legendre.leggauss(tp + 1)[0])
            U = np.einsum("ab,cbv->cav", W, U)
            if sst:
                tk, tw, tn = (np.einsum("ab,cb->ca", W, x) for x in (tk, tw, tn))
                wd = np.einsum("ab,cb->ca", W, wd)
            cur = tp
        mesh = Mesh.from_case(case_for_order(tp))
        if mfs_cache is None:
            mfs_cache = metric_flux_scale(mesh)
        mesh.extras["mfs"] = np.broadcast_to(mfs_cache, (mesh.N, mesh.S)) if mfs_cache.shape[1] in (1, mesh.S) \
            else np.tile(mfs_cache, (1, -(-mesh.S // mfs_cache.shape[1])))[:, :mesh.S]
        s = Solver(mesh, U, mu, TurbState(tk, tw, tn) if sst else None, wd, inviscid_only, 0.0)
        states[f"U_start_p{tp}"] = s.U.copy()
        phase_max, phase_tol = max_iter // len(orders), tol * (10 ** (order - tp))
        init, converged = None, False
        for i in range(phase_max):
            res = s.step()
            final = res
            total += 1
            step_order.append(tp)
            step_res.append(res)
            if init is None:
                init = res
            if res < phase_tol:
                converged = True
                break
            if tp < order and i >= 20 and init > 0 and init / max(res, 1e-30) >= 1e2:
                break
        U = s.U
        states[f"U_end_p{tp}"] = U.copy()
        if sst:
            tk, tw, tn = s.turb.k, s.turb.w, s.turb.nut
            states[f"k_end_p{tp}"], states[f"w_end_p{tp}"], states[f"nut_end_p{tp}"] = tk.copy(), tw.copy(), tn.copy()
        if tp == order and converged:
            return step_order, step_res, states, (True, total, final)
    return step_order, step_res, states, (False, total, final)


def case_from_prefix(case, prefix):
    """The tables a continuation fixture stores for one phase (keys
    ``<prefix><name>``), as a case of their own."""
    return {k[len(prefix):]: case[k] for k in case if k.startswith(prefix)}


def load_case(path):
    """Mesh + Solver from a golden .npz."""
    z = np.load(path, allow_pickle=False)
    case = {k: z[k] for k in z.files}
    m = Mesh.from_case(case)
    turb = None
    wd = None
    if str(case["turb"]) == "SST":
        turb = TurbState(case["k0"].copy(), case["omega0"].copy(), case["nu_t0"].copy())
        wd = case["wall_distance"]
    s = Solver(m, case["U0"].copy(), float(case["mu"]), turb, wd, bool(case["inviscid_only"]),
               float(case["global_dt_factor"]))
    if "time_scheme" in case:
        s.time_scheme = str(case["time_scheme"])
        s.dt_step = float(case["dt_step"])
        s.dual_time_inner_iter = int(case["dual_time_inner_iter"])
    return case, m, s
