"""ORACLE — test infrastructure only.

A numpy restatement of the differentiated MPS path, the checker of the
device adjoint (wqc_adjoint_forward / wqc_adjoint_backward).  The reference
has no adjoint; what is differentiated is its forward path: one-qubit gates
(src/tn/mps.rs:333-351), adjacent two-site applies with the 4x4 on theta
(mps.rs:377-429, 833-866) and the truncated split (mps.rs:1124-1171:
exact SVD, kept chi by retained_chi, svd_guard.rs:25-35, L = U sqrt(S),
R = sqrt(S) V^H, no renormalisation), then f = sum_t Re(c_t) <psi|P_t|psi>
(src/expectation.rs:98-200).

The backward pass is the complex SVD's reverse mode over the full thin SVD,
with the cotangents of the dropped singular vectors zero, which carries the
truncation term (kept-dropped couplings 1/(s_j^2 - s_i^2)); every
1/(s_j^2 - s_i^2) is Lorentzian-broadened, (s_j^2 - s_i^2) / ((s_j^2 -
s_i^2)^2 + eps), eps = LORENTZ_EPS * s_max^4.  Columns whose singular value
is at rounding level join the null-space projectors.

Only circuits of one-qubit gates and adjacent CNOT/CZ are handled here (the
ansatz shape of the differentiation workload); the device version takes any
gate list.
"""
from __future__ import annotations

import numpy as np

import dense as D

CUTOFF = 1e-12  # SINGULAR_CUTOFF, svd_guard.rs:12
LORENTZ_EPS = 1e-24  # relative to s_max^4
NULL_REL = 1e-14  # singular values below NULL_REL * s_max count as null directions


def _cnot4():
    m = np.zeros((2, 2, 2, 2), dtype=complex)
    m[0, 0, 0, 0] = m[0, 1, 0, 1] = m[1, 0, 1, 1] = m[1, 1, 1, 0] = 1
    return m


def _cz4():
    m = np.zeros((2, 2, 2, 2), dtype=complex)
    m[0, 0, 0, 0] = m[0, 1, 0, 1] = m[1, 0, 1, 0] = 1
    m[1, 1, 1, 1] = -1
    return m


def effective(u4, ctrl_is_first: bool) -> np.ndarray:
    """The 4x4 on theta[a][s][t][b] as [(so, to), (si, ti)] (mps.rs:396-421)."""
    out = np.zeros((4, 4), dtype=complex)
    for so in range(2):
        for to in range(2):
            for si in range(2):
                for ti in range(2):
                    if ctrl_is_first:
                        out[so * 2 + to, si * 2 + ti] = u4[so, to, si, ti]
                    else:
                        out[so * 2 + to, si * 2 + ti] = u4[to, so, ti, si]
    return out


def d_unary(kind: int, theta: float) -> np.ndarray:
    """d/dtheta of the rotation matrices of gates.rs:10-66."""
    s, c = np.sin(theta / 2.0), np.cos(theta / 2.0)
    if kind == D.RX:
        return 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]])
    if kind == D.RY:
        return 0.5 * np.array([[-s, -c], [c, -s]])
    if kind == D.RZ:
        return 0.5 * np.array([[complex(-s, -c), 0], [0, complex(-s, c)]])
    return np.zeros((2, 2), dtype=complex)


def ops_of(gates):
    """(kind, site(s), matrix, gate index) per operation; adjacent 2q only."""
    ops = []
    for i, g in enumerate(gates):
        k = int(g["kind"])
        if k in (D.CNOT, D.CZ):
            c, t = int(g["q0"]), int(g["q1"])
            if abs(c - t) != 1:
                raise ValueError("the numpy adjoint takes adjacent two-qubit gates only")
            u4 = _cnot4() if k == D.CNOT else _cz4()
            ops.append(("2q", min(c, t), effective(u4, c < t), i))
        elif k in (D.MEASURE, D.RESET, D.IF):
            continue
        else:
            ops.append(("1q", int(g["q0"]), D.unary(k, float(g["angle"])), i))
    return ops


def split(theta_m, chi_max):
    u, s, vh = np.linalg.svd(theta_m, full_matrices=False)
    rank = int(np.sum(s > CUTOFF))
    k = min(max(rank, 1), chi_max, theta_m.shape[0], theta_m.shape[1])
    return u, s, vh, k


def forward(n, chi_max, gates, keep=False):
    sites = [np.array([1.0, 0.0], dtype=complex).reshape(1, 2, 1) for _ in range(n)]
    tape = []
    for kind, p, mat, gi in ops_of(gates):
        if kind == "1q":
            if keep:
                tape.append((kind, p, mat, gi, sites[p].copy()))
            sites[p] = np.einsum("xs,asb->axb", mat, sites[p])
        else:
            a, b = sites[p], sites[p + 1]
            th = np.einsum("asg,gtb->astb", a, b)
            dl, dr = a.shape[0], b.shape[2]
            th = np.einsum("xy,ayb->axb", mat, th.reshape(dl, 4, dr)).reshape(2 * dl, 2 * dr)
            u, s, vh, k = split(th, chi_max)
            if keep:
                tape.append((kind, p, mat, gi, (a.copy(), b.copy(), th, u, s, vh, k)))
            d = np.sqrt(s[:k])
            sites[p] = (u[:, :k] * d).reshape(dl, 2, k)
            sites[p + 1] = (d[:, None] * vh[:k]).reshape(k, 2, dr)
    return sites, tape


def dense_of(sites):
    st = np.ones((1, 1), dtype=complex)
    for s in sites:
        st = np.einsum("xa,asb->sxb", st, s).reshape(-1, s.shape[2])
    return st[:, 0]


def pauli_apply(state, label):
    n = len(label)
    idx = np.arange(1 << n)
    out = state.copy()
    for q in range(n):
        ch = label[n - 1 - q]
        bit = (idx >> q) & 1
        if ch == "X":
            out = out[idx ^ (1 << q)]
        elif ch == "Y":
            out = out[idx ^ (1 << q)] * np.where(bit == 1, 1j, -1j)
        elif ch == "Z":
            out = out * np.where(bit == 1, -1.0, 1.0)
    return out


def value(n, chi_max, gates, labels, coeffs):
    sites, _ = forward(n, chi_max, gates)
    psi = dense_of(sites)
    return sum(np.real(c) * np.real(np.vdot(psi, pauli_apply(psi, lab))) for lab, c in zip(labels, coeffs))


def site_cotangents(sites, psibar):
    """A_bar_q[a, s, b] = sum_x psibar[x] conj(d psi[x] / d A_q[a, s, b])."""
    n = len(sites)
    left = [np.ones((1, 1), dtype=complex)]  # [prefix, a]
    for q in range(n - 1):
        s = sites[q]
        left.append(np.einsum("xa,asb->sxb", left[-1], s).reshape(-1, s.shape[2]))
    right = [None] * n
    right[n - 1] = np.ones((1, 1), dtype=complex)  # [b, suffix]
    for q in range(n - 1, 0, -1):
        s = sites[q]
        right[q - 1] = np.einsum("asb,by->ays", s, right[q]).reshape(s.shape[0], -1)
    out = []
    for q in range(n):
        pre, suf = left[q].shape[0], right[q].shape[1]
        pb = psibar.reshape(suf, 2, pre)  # basis = suffix * 2^(q+1) + s * 2^q + prefix
        out.append(np.einsum("ysx,xa,by->asb", pb, left[q].conj(), right[q].conj()))
    return out


def svd_backward(u, s, vh, k, ubar_k, sbar_k, vbar_k):
    """theta_bar from the cotangents of the kept columns (U_k, s_k, V_k)."""
    smax = s[0] if s.size else 0.0
    r = int(np.sum(s > NULL_REL * smax)) if smax > 0 else 0
    r = max(r, k)
    U, V, sv = u[:, :r], vh[:r].conj().T, s[:r]
    Ub = np.zeros((u.shape[0], r), dtype=complex)
    Vb = np.zeros((V.shape[0], r), dtype=complex)
    sb = np.zeros(r)
    Ub[:, :k], Vb[:, :k], sb[:k] = ubar_k, vbar_k, sbar_k
    M = U.conj().T @ Ub
    N = V.conj().T @ Vb
    d2 = sv[None, :] ** 2 - sv[:, None] ** 2  # s_j^2 - s_i^2
    F = d2 / (d2 ** 2 + LORENTZ_EPS * smax ** 4)
    np.fill_diagonal(F, 0.0)
    G = F * ((M - M.conj().T) * sv[None, :] + sv[:, None] * (N - N.conj().T))
    inv = np.where(sv > 0, 1.0 / np.where(sv > 0, sv, 1.0), 0.0)
    G[np.diag_indices(r)] += sb + 1j * np.imag(np.diag(M) - np.diag(N)) * inv / 2.0
    tb = U @ G @ V.conj().T
    q1 = Ub * inv[None, :]
    tb += (q1 - U @ (U.conj().T @ q1)) @ V.conj().T
    q2 = Vb * inv[None, :]
    tb += U @ (q2 - V @ (V.conj().T @ q2)).conj().T
    return tb


def gradient(n, chi_max, gates, labels, coeffs):
    """(f, df/dangle per gate): reverse sweep over the stored forward."""
    sites, tape = forward(n, chi_max, gates, keep=True)
    psi = dense_of(sites)
    f = sum(np.real(c) * np.real(np.vdot(psi, pauli_apply(psi, lab))) for lab, c in zip(labels, coeffs))
    psibar = sum(2.0 * np.real(c) * pauli_apply(psi, lab) for lab, c in zip(labels, coeffs))
    bars = site_cotangents(sites, psibar)
    grad = np.zeros(len(gates))
    for kind, p, mat, gi, saved in reversed(tape):
        if kind == "1q":
            before = saved
            g = gates[gi]
            du = d_unary(int(g["kind"]), float(g["angle"]))
            grad[gi] += np.real(np.vdot(bars[p], np.einsum("xs,asb->axb", du, before)))
            bars[p] = np.einsum("sx,asb->axb", mat.conj(), bars[p])
        else:
            a, b, th, u, s, vh, k = saved
            dl, dr = a.shape[0], b.shape[2]
            lbar = bars[p].reshape(2 * dl, k)
            rbar = bars[p + 1].reshape(k, 2 * dr)
            d = np.sqrt(s[:k])
            uk, vk = u[:, :k], vh[:k].conj().T
            ubar = lbar * d[None, :]
            vbar = rbar.conj().T * d[None, :]
            sbar = (np.real(np.sum(uk.conj() * lbar, axis=0)) + np.real(np.sum(rbar.T * vk, axis=0))) / (2 * d)
            tb = svd_backward(u, s, vh, k, ubar, sbar, vbar)
            tb0 = np.einsum("yx,ayb->axb", mat.conj(), tb.reshape(dl, 4, dr)).reshape(2 * dl, 2 * dr)
            kin = a.shape[2]
            am, bm = a.reshape(2 * dl, kin), b.reshape(kin, 2 * dr)
            bars[p] = (tb0 @ bm.conj().T).reshape(dl, 2, kin)
            bars[p + 1] = (am.conj().T @ tb0).reshape(kin, 2, dr)
    return f, grad
