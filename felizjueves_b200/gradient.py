"""The J and K terms of the nuclear gradient of G, on the Fock build.

    jk_derivatives(basis, D) -> (vj1, vk1)        3 x n x n each
    gradient_jk(basis, D, nuclei) -> (grad_J, grad_K)   n_atoms x 3 each

The derivative integrals come from the ordinary build by the Cartesian
shift identity: on the electron coordinate of a function of shell A,

    d/dx [x_A^i e^(-alpha r_A^2)] = -2 alpha x_A^(i+1) e^(...) + i x_A^(i-1) e^(...)

so (d_x a b|c d) is a combination of integrals over the shell A+ (l + 1,
coefficients c (-2 alpha)) and A- (l - 1, coefficients c).  The build runs
once over the basis extended by every A+ and A-, with the density D on the
original block and zero elsewhere: its J and K rows of the shifted functions
are sum_kl (A+- j|k l) D_lk and sum_jk (A+- j|k l) D_jk, and

    vj1[x, i, j] = -(J[i+1_x, j] + i_x J[i-1_x, j])
    vk1[x, i, l] = -(K[i+1_x, l] + i_x K[i-1_x, l])

-- PySCF's grad.rhf.get_jk convention over libcint's int2e_ip1, which the
reference's gradient fixtures record (its own path: gradient/kernel_gf.py).
Per atom A, over the AOs i on A:

    grad_J[A] = 2 sum_(i on A) sum_j vj1[:, i, j] D[i, j]
    grad_K[A] = 2 sum_(i on A) sum_j (-1/2) vk1[:, i, j] D[i, j]

The shifted shells reach l + 1, so the basis may hold shells to l = 2 (the
kernels are compiled to l = 3).  `jk=` injects the (J, K) evaluator of the
extended basis (the reference's drivers take `eri=` the same way); the
default is the GPU build, unscreened (tau = 0) unless `tau` is given.
"""

from __future__ import annotations

import numpy as np

from .fock import FockEngine, _checked_density, _checked_nuclei
from .shell import Basis, Shell, cartesians


def extended_basis(basis: Basis):
    """(B_ext, up, dn): the basis followed by every shell at l + 1 (c times
    -2 alpha) and every shell of l >= 1 at l - 1; up[s] / dn[s] the extended
    shell index of shell s's shifts (dn[s] None for s shells)."""
    sh = list(basis.shells)
    if any(s.l > 2 for s in sh):
        raise ValueError("the gradient's shifted shells reach l + 1: shells to l = 2 only")
    ext = list(sh)
    up, dn = [], []
    for s in sh:
        up.append(len(ext))
        ext.append(Shell(s.l + 1, s.centre, s.exponents,
                         tuple(-2.0 * a * c for a, c in zip(s.exponents, s.coefficients))))
    for s in sh:
        if s.l >= 1:
            dn.append(len(ext))
            ext.append(Shell(s.l - 1, s.centre, s.exponents, s.coefficients))
        else:
            dn.append(None)
    return Basis(tuple(ext)), up, dn


def _gpu_jk(tau: float, device: int):
    def jk(B, D):
        eng = FockEngine(B, device)
        eng.plan(D, tau, 4, export=False)
        J, K, _ = eng.build_host(D)
        return J, K
    return jk


def jk_derivatives(basis: Basis, D, *, tau: float = 0.0, device: int = 0, jk=None):
    """(vj1, vk1) of the symmetric density D (module docstring)."""
    D = _checked_density(basis, D)
    B, up, dn = extended_basis(basis)
    n, m = basis.n_ao, B.n_ao
    Dx = np.zeros((m, m))
    Dx[:n, :n] = D
    J, K = (jk or _gpu_jk(tau, device))(B, Dx)
    vj1 = -_shift_rows(basis, B, up, dn, J)
    vk1 = -_shift_rows(basis, B, up, dn, K)
    return vj1, vk1


def _shift_rows(basis: Basis, B: Basis, up, dn, M: np.ndarray) -> np.ndarray:
    """out[x, i, :] = M[i+1_x, :n] + i_x M[i-1_x, :n] over the original AOs
    i: the electron-coordinate derivative of the bra function, as rows of a
    matrix over the extended basis."""
    n = basis.n_ao
    out = np.zeros((3, n, n))
    for s, shell in enumerate(basis.shells):
        iu = {c: B.offsets[up[s]] + k for k, c in enumerate(cartesians(shell.l + 1))}
        idn = ({c: B.offsets[dn[s]] + k for k, c in enumerate(cartesians(shell.l - 1))}
               if dn[s] is not None else {})
        for r, comp in enumerate(cartesians(shell.l)):
            i = basis.offsets[s] + r
            for x in range(3):
                cp = list(comp)
                cp[x] += 1
                v = M[iu[tuple(cp)], :n].copy()
                if comp[x] > 0:
                    cm = list(comp)
                    cm[x] -= 1
                    v += comp[x] * M[idn[tuple(cm)], :n]
                out[x, i] = v
    return out


def _gpu_onee(device: int):
    def onee(B, nuclei):
        eng = FockEngine(B, device)
        S, T, V, _ = eng.one_electron(nuclei, want=("S", "T", "V"))
        return S.cpu().numpy(), T.cpu().numpy(), V.cpu().numpy()
    return onee


def one_electron_derivatives(basis: Basis, nuclei, *, device: int = 0, onee=None):
    """libcint's int1e_ipovlp, int1e_ipkin, int1e_ipnuc (3 x n x n) and
    int1e_iprinv at each nucleus (n_atoms x 3 x n x n): <d_x i|O|j> with d_x
    on the electron coordinate of i, from the one-electron matrices of the
    shift-extended basis (rinv at nucleus C: V of one charge -1 there)."""
    nuc = _checked_nuclei(nuclei)
    B, up, dn = extended_basis(basis)
    ev = onee or _gpu_onee(device)
    S, T, V = ev(B, nuc)
    ipovlp = _shift_rows(basis, B, up, dn, S)
    ipkin = _shift_rows(basis, B, up, dn, T)
    ipnuc = _shift_rows(basis, B, up, dn, V)
    iprinv = np.stack([_shift_rows(basis, B, up, dn, ev(B, [(-1.0, c)])[2]) for _, c in nuc])
    return ipovlp, ipkin, ipnuc, iprinv


def nuclear_repulsion_gradient(nuclei) -> np.ndarray:
    """d V_nn / d R_A = -sum_B Z_A Z_B (R_A - R_B) / |R_A - R_B|^3."""
    nuc = _checked_nuclei(nuclei)
    g = np.zeros((len(nuc), 3))
    for a, (za, ca) in enumerate(nuc):
        for b, (zb, cb) in enumerate(nuc):
            if a != b:
                d = np.subtract(ca, cb)
                g[a] -= za * zb * d / np.linalg.norm(d) ** 3
    return g


def rhf_gradient(basis: Basis, nuclei, D, W, *, tau: float = 0.0, device: int = 0, jk=None,
                 onee=None) -> dict:
    """The closed-shell SCF nuclear gradient of density D and energy-
    weighted density W = 2 sum_occ e_i C_i C_i^T, per term (PySCF's
    grad.rhf.grad_elec + grad_nuc, which the reference's fixtures record):

        h[A]   = sum_ij dh^A_ij D_ij,  dh^A = v + v^T,
                 v = -Z_A rinv'_A, rows of A's AOs plus -(ipkin + ipnuc)
        s[A]   = 2 sum_(i on A) sum_j ipovlp[:, i, j] W_ij
        j[A], k[A]  as gradient_jk
        nuc[A] the nuclear repulsion's
    and their sum `total` (n_atoms x 3 each)."""
    nuc = _checked_nuclei(nuclei)
    D = _checked_density(basis, D)
    W = np.asarray(W, np.float64)
    atoms = ao_atoms(basis, nuc)
    ipovlp, ipkin, ipnuc, iprinv = one_electron_derivatives(basis, nuc, device=device, onee=onee)
    h1 = -(ipkin + ipnuc)
    gh = np.zeros((len(nuc), 3))
    gs = np.zeros((len(nuc), 3))
    for a, (za, _) in enumerate(nuc):
        v = -za * iprinv[a]
        rows = atoms == a
        v[:, rows] += h1[:, rows]
        gh[a] = np.einsum("xij,ij->x", v + v.transpose(0, 2, 1), D)
        gs[a] = 2.0 * np.einsum("xij,ij->x", ipovlp[:, rows], W[rows])
    gj, gk = gradient_jk(basis, D, nuc, tau=tau, device=device, jk=jk)
    gn = nuclear_repulsion_gradient(nuc)
    return {"h": gh, "s": gs, "j": gj, "k": gk, "nuc": gn, "total": gh + gs + gj + gk + gn}


def ao_atoms(basis: Basis, nuclei) -> np.ndarray:
    """The atom (index into nuclei) of every AO: its shell's centre."""
    nuc = _checked_nuclei(nuclei)
    out = []
    for s in basis.shells:
        hit = [k for k, (_, c) in enumerate(nuc) if c == tuple(float(x) for x in s.centre)]
        if len(hit) != 1:
            raise ValueError(f"a shell at {s.centre} sits on {len(hit)} nuclei, not one")
        out.extend([hit[0]] * s.n_cart)
    return np.asarray(out, np.int32)


def gradient_jk(basis: Basis, D, nuclei, *, tau: float = 0.0, device: int = 0, jk=None):
    """(grad_J, grad_K), each n_atoms x 3 (module docstring)."""
    D = _checked_density(basis, D)
    vj1, vk1 = jk_derivatives(basis, D, tau=tau, device=device, jk=jk)
    atoms = ao_atoms(basis, nuclei)
    gj = np.zeros((len(nuclei), 3))
    gk = np.zeros((len(nuclei), 3))
    for i, a in enumerate(atoms):
        gj[a] += 2.0 * vj1[:, i, :] @ D[i, :]
        gk[a] += 2.0 * (-0.5 * vk1[:, i, :]) @ D[i, :]
    return gj, gk
