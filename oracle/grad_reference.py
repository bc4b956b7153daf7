"""FP64 reference gradients of exciton energies -- TEST INFRASTRUCTURE ONLY.

The reference (Xatu v1.3.1) has no derivative code.  This module restates its
build+solve path once more, in torch (complex128 / float64), so that
reverse-mode automatic differentiation gives the exact gradient of the
reference's energies with respect to the hopping matrices H(R), r0, eps_m and
eps_s.  It is the "FP64 reference gradient" the engine's hand-written adjoint
is checked against; it is itself checked against central finite differences
of the C/numpy oracle (tests/test_grad_reference.py).

Steps restated (each follows the same reference lines as oracle/oracle.py and
oracle/xatu_oracle.c):
  * Struve H0 (ExcitonTB.cpp:306-337): same branches and the same per-element
    series truncation, so that its derivative is the derivative of the
    reference's approximation; Y0 with dY0/dx = -Y1;
  * Keldysh / Coulomb potentials and keldyshFT (ExcitonTB.cpp:347-426);
  * motif lattice Fourier transform, upper triangle + conjugate (:438-476);
  * Bloch Hamiltonian with the triangular symmetrisation, Loewdin (SystemTB.cpp:60-156),
    eigh, fixGlobalPhase (ExcitonTB.cpp:673-683);
  * BShamiltonian: real-space or reciprocal-space direct term, exchange,
    upper triangle, H = U + U^H with the diagonal (ExcitonTB.cpp:520-621, 840-921);
  * eigvalsh of H.
Sizes: for the small systems of the tests (N up to a few hundred).
"""
from __future__ import annotations

import numpy as np
import torch

from . import oracle as O

PI = 3.141592653589793
EC = 1.6021766e-19
EPS0 = 8.8541878e-12


def struve_h0(x: torch.Tensor) -> torch.Tensor:
    """ExcitonTB::STVH0 (ExcitonTB.cpp:306-337) on a float64 tensor, per-element truncation."""
    out = torch.zeros_like(x)
    small = x <= 20.0
    if bool(small.any()):
        xs = x[small]
        s = torch.ones_like(xs)
        r = torch.ones_like(xs)
        active = torch.ones_like(xs, dtype=torch.bool)
        for k in range(1, 61):
            d = 2.0 * k + 1.0
            rn = -r * xs / d * xs / d
            r = torch.where(active, rn, r)
            s = torch.where(active, s + rn, s)
            active = active & ~(rn.abs() < s.abs() * 1.0e-12)
            if not bool(active.any()):
                break
        out = out.index_put((small,), 2.0 * xs / PI * s)
    large = ~small
    if bool(large.any()):
        xl = x[large]
        km = torch.where(xl >= 50.0, torch.full_like(xl, 25.0), torch.floor(0.5 * (xl.detach() + 1.0)))
        s = torch.ones_like(xl)
        r = torch.ones_like(xl)
        active = torch.ones_like(xl, dtype=torch.bool)
        for k in range(1, int(km.max().item()) + 1):
            act = active & (k <= km)
            u = (2.0 * k - 1.0) / xl
            rn = -r * (u * u)
            r = torch.where(act, rn, r)
            s = torch.where(act, s + rn, s)
            active = act & ~(rn.abs() < s.abs() * 1.0e-12)
        t = 4.0 / xl
        t2 = t * t
        p0 = ((((-.37043e-5 * t2 + .173565e-4) * t2 - .487613e-4) * t2 + .17343e-3) * t2 - 0.1753062e-2) * t2 + \
            .3989422793
        q0 = t * (((((.32312e-5 * t2 - 0.142078e-4) * t2 + 0.342468e-4) * t2 - 0.869791e-4) * t2 +
                   0.4564324e-3) * t2 - 0.0124669441)
        ta0 = xl - 0.25 * PI
        by0 = 2.0 / torch.sqrt(xl) * (p0 * torch.sin(ta0) + q0 * torch.cos(ta0))
        out = out.index_put((large,), 2.0 / (PI * xl) * s + by0)
    return out


class _Y0(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        ctx.save_for_backward(x)
        return torch.special.bessel_y0(x)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return -g * torch.special.bessel_y1(x)


def keldysh(r: torch.Tensor, r0, eps_m, eps_s, regularization: float, rcut: float) -> torch.Tensor:
    """ExcitonTB::keldysh (ExcitonTB.cpp:347-366) for a tensor of distances (no gradient through r)."""
    eps_bar = (eps_m + eps_s) / 2
    pref = EC / (8e-10 * EPS0 * eps_bar * r0)
    rr = torch.where(r == 0, torch.full_like(r, regularization), r.abs())
    x = rr / r0
    v = pref * (struve_h0(x) - _Y0.apply(x))
    return torch.where((r != 0) & (r > rcut), torch.zeros_like(v), v)


def coulomb(r: torch.Tensor, regularization: float, rcut: float) -> torch.Tensor:
    """ExcitonTB::coulomb (ExcitonTB.cpp:374-381)."""
    r = r.abs()
    safe = torch.where(r == 0, torch.ones_like(r), r)
    v = torch.where(r != 0, EC / (4e-10 * PI * EPS0 * safe), torch.full_like(r, EC * 1e10 / (4 * PI * EPS0 *
                                                                                               regularization)))
    return torch.where(r > rcut, torch.zeros_like(v), v)


class TorchExciton:
    """The path of an initialised OracleExciton as a differentiable function of
    (H(R), r0, eps_m, eps_s)."""

    def __init__(self, ex: "O.OracleExciton"):
        self.ex = ex
        s = ex.system
        self.na = s.natoms
        self.norb = s.basisdim
        self.atom_of = np.repeat(np.arange(s.natoms), s.orb_per_atom)
        self.tau = torch.tensor(s.motif[:, :3], dtype=torch.float64)
        self.kpts = torch.tensor(ex.kpoints, dtype=torch.float64)
        self.cellsR = torch.tensor(s.cells_h, dtype=torch.float64)
        self.cells = torch.tensor(ex.cells, dtype=torch.float64)
        self.mesh = torch.tensor(ex.mesh, dtype=torch.float64)
        self.Q = torch.tensor(ex.Q, dtype=torch.float64)
        self.S = None
        if s.overlap is not None and len(s.overlap):
            self.S = torch.tensor(np.asarray(s.overlap), dtype=torch.complex128)
        nk = ex.kpoints.shape[0]
        self.bk = torch.tensor(ex.basis_k, dtype=torch.long)
        self.bc = torch.tensor(ex.basis_c, dtype=torch.long)
        self.bv = torch.tensor(ex.basis_v, dtype=torch.long)
        # real-space mesh index of k_j - k_i (findEquivalentPointBZ, Lattice.cpp:251-279)
        if ex.mode == "realspace":
            idx = np.zeros((nk, nk), dtype=np.int64)
            for i in range(nk):
                for j in range(nk):
                    idx[i, j] = O.find_equivalent_point(s.recip, ex.inv_recip, ex.ncell * ex.factor,
                                                        ex.kpoints[j] - ex.kpoints[i])
            self.qidx = torch.tensor(idx)
        self.G = torch.tensor(ex.G, dtype=torch.float64)

    # ------------------------------------------------------------------ stages
    def bands(self, HR: torch.Tensor, shift: torch.Tensor):
        ex, s = self.ex, self.ex.system
        k = self.kpts + shift[None, :]
        ph = torch.exp(1j * (k @ self.cellsR.T))                      # nk x nR
        H = torch.einsum("kr,rij->kij", ph, HR)
        if s.is_triangular:
            H = H - torch.diag_embed(torch.diagonal(H, dim1=1, dim2=2) / 2)
            H = H + H.conj().transpose(1, 2)
        if self.S is not None:
            Sk = torch.einsum("kr,rij->kij", ph, self.S)
            if s.is_triangular:
                Sk = Sk - torch.diag_embed(torch.diagonal(Sk, dim1=1, dim2=2) / 2)
                Sk = Sk + Sk.conj().transpose(1, 2)
            if s.is_au:
                H = H * 27.2
            w, u = torch.linalg.eigh(Sk)
            X = (u * (1.0 / torch.sqrt(w))[:, None, :]) @ u.conj().transpose(1, 2)
            H = X @ H @ X
        w, U = torch.linalg.eigh(H)
        ssum = U.sum(dim=1)                                            # nk x norb
        zeta = ssum.conj() / ssum.abs()
        C = U * zeta[:, None, :]
        bl = torch.tensor(ex.band_list, dtype=torch.long)
        return w[:, bl], C[:, :, bl].transpose(1, 2)                   # nk x nb, nk x nb x norb

    def pair_potential(self, kind: str, r0, eps_m, eps_s, q: torch.Tensor) -> torch.Tensor:
        """motifFourierTransform (ExcitonTB.cpp:438-476) for the rows of q."""
        ex, na = self.ex, self.na
        rcut = ex.system.a * ex.cutoff + 1e-5
        out = torch.zeros((q.shape[0], na, na), dtype=torch.complex128)
        ph = torch.exp(1j * (q @ self.cells.T))                        # nq x ncells
        for a in range(na):
            for b in range(a, na):
                d = torch.linalg.norm(self.cells + (self.tau[a] - self.tau[b])[None, :], dim=1)
                v = keldysh(d, r0, eps_m, eps_s, ex.regularization, rcut) if kind == "keldysh" else \
                    coulomb(d, ex.regularization, rcut)
                f = (ph * v[None, :].to(torch.complex128)).sum(dim=1) / ex.total_cells
                out = out.index_put((torch.arange(q.shape[0]), torch.tensor(a), torch.tensor(b)), f)
                if b != a:
                    out = out.index_put((torch.arange(q.shape[0]), torch.tensor(b), torch.tensor(a)), f.conj())
        return out

    def keldysh_ft(self, q: torch.Tensor, r0, eps_m, eps_s) -> torch.Tensor:
        """ExcitonTB::keldyshFT (ExcitonTB.cpp:410-426) for q of shape (..., 3)."""
        ex, s = self.ex, self.ex.system
        eps_bar = (eps_m + eps_s) / 2
        eps = float(np.linalg.norm(s.recip[0])) / ex.total_cells
        qn = torch.linalg.norm(q, dim=-1)
        safe = torch.where(qn < eps, torch.ones_like(qn), qn)
        pot = torch.where(qn < eps, torch.zeros_like(qn), 1.0 / (safe * (1 + r0 * safe)))
        return pot * EC * 1e10 / (2 * EPS0 * eps_bar * s.area * ex.total_cells)

    def hamiltonian(self, HR, r0, eps_m, eps_s) -> torch.Tensor:
        ex = self.ex
        e0, C0 = self.bands(HR, torch.zeros(3, dtype=torch.float64))
        if float(np.linalg.norm(ex.Q)) != 0:
            eQ, CQ = self.bands(HR, self.Q)
        else:
            eQ, CQ = e0, C0
        bk, bc, bv = self.bk, self.bc, self.bv
        ci = CQ[bk, bc]                         # N x norb: conduction at k (+Q)
        vi = C0[bk, bv]                         # N x norb: valence at k
        na = self.na
        A = torch.zeros((self.norb, na), dtype=torch.complex128)
        A[np.arange(self.norb), self.atom_of] = 1.0
        # rho1[i,j,a] = sum_{o in a} conj(c_i) c_j ; rho2[i,j,b] = sum_{o in b} conj(v_j) v_i
        rho1 = torch.einsum("io,jo,oa->ija", ci.conj(), ci, A)
        rho2 = torch.einsum("jo,io,oa->ija", vi.conj(), vi, A)
        L = torch.einsum("io,io,oa->ia", ci.conj(), vi, A)              # exchange factor of state i
        if ex.mode == "realspace":
            V = self.pair_potential(ex.potential, r0, eps_m, eps_s, self.mesh)
            Vij = V[self.qidx[bk][:, bk]]                                  # N x N x na x na
            D = torch.einsum("ija,ijab,ijb->ij", rho1, Vij, rho2)
            X = torch.zeros_like(D)
            if ex.exchange:
                VQ = self.pair_potential(ex.exchange_potential, r0, eps_m, eps_s, self.Q[None, :])[0]
                X = torch.einsum("ia,ab,jb->ij", L, VQ, L.conj())
        else:
            kk = self.kpts[bk]                                             # N x 3
            dk = kk[:, None, :] - kk[None, :, :]                           # k_i - k_j
            D = torch.zeros((len(bk), len(bk)), dtype=torch.complex128)
            X = torch.zeros_like(D)
            for g in range(self.G.shape[0]):
                q = dk + self.G[g][None, None, :]
                ph = torch.exp(1j * torch.einsum("ijx,ax->ija", q, self.tau))
                Ic = (rho1 * ph).sum(-1)
                Iv = (rho2.conj() * ph).sum(-1)
                D = D + Ic * Iv.conj() * self.keldysh_ft(q, r0, eps_m, eps_s)
                if ex.exchange:
                    qx = self.Q + self.G[g]
                    phx = torch.exp(1j * (self.tau @ qx))
                    Icx = (L * phx[None, :]).sum(-1)
                    X = X + Icx[:, None] * Icx.conj()[None, :] * self.keldysh_ft(qx[None, :], r0, eps_m, eps_s)[0]
        M = -(D - X)
        U = torch.triu(M, diagonal=1)
        ec = eQ[bk, bc]
        ev = e0[bk, bv]
        d = ex.scissor + ec - ev - torch.diagonal(D - X).real
        return U + U.conj().T + torch.diag(d.to(torch.complex128))

    def energies(self, HR, r0, eps_m, eps_s) -> torch.Tensor:
        return torch.linalg.eigvalsh(self.hamiltonian(HR, r0, eps_m, eps_s))


def reference_gradients(ex: "O.OracleExciton", nstates: int) -> dict:
    """Energies of the lowest ``nstates`` excitons and their gradients with respect to H(R)
    (complex: d/dRe + i d/dIm, shape nstates x nR x norb x norb), r0, eps_m and eps_s."""
    te = TorchExciton(ex)
    s = ex.system
    HR = torch.tensor(s.hamiltonian, dtype=torch.complex128, requires_grad=True)
    r0 = torch.tensor(ex.r0, dtype=torch.float64, requires_grad=True)
    em = torch.tensor(ex.eps_m, dtype=torch.float64, requires_grad=True)
    es = torch.tensor(ex.eps_s, dtype=torch.float64, requires_grad=True)
    E = te.energies(HR, r0, em, es)
    out = {"energies": E[:nstates].detach().numpy().copy(),
           "hamiltonian": np.zeros((nstates,) + tuple(HR.shape), dtype=np.complex128),
           "r0": np.zeros(nstates), "eps_m": np.zeros(nstates), "eps_s": np.zeros(nstates)}
    for n in range(nstates):
        g = torch.autograd.grad(E[n], [HR, r0, em, es], retain_graph=True, allow_unused=True)
        out["hamiltonian"][n] = g[0].numpy() if g[0] is not None else 0
        out["r0"][n] = float(g[1]) if g[1] is not None else 0.0
        out["eps_m"][n] = float(g[2]) if g[2] is not None else 0.0
        out["eps_s"][n] = float(g[3]) if g[3] is not None else 0.0
    return out
