"""GPU-resident projected-HF optimiser step: EandG with every array on the device, and an L-BFGS loop.

``DeviceEandG`` is the reference driver's ``EandG`` (PHF.py:55-91) with the parameters, the
determinant, the grid accumulators and the gradient kept on the GPU.  For the real parameter vector
x = [Re z; Im z] of the (M - N) x N Thouless matrix z in the Ref-MO basis it computes

    sol = P(z)                    FrozenProj, CmplxConj = 0, SzProj, RHFProj (PHF.py:58-66, :133-151)
    C   = Ref [I; sol]            the determinant buildhsg forms from (Ref, Z) (PHFTools.f90:69-77)
    H, S, Yg, Yr                  one pass of the plan (phf_plan_eval_device_async, no host sync)
    E0, f                         EigenSolver + VecDecomp (PHFTools.py:8-26) of the nci x nci Hmat, Smat
    G   = LocalG[N:, :N]          (PHFTools.f90:203-247) = [Ref^H (sum f*f Yg - E0 sum f*f Yr) / sum f*f S][N:, :]
    g   = [Re P(G); Im P(G)]      (PHF.py:78-90)

and returns (E0, g) as device tensors.  ``host(x)`` is the same call with numpy in and out (one
host -> device copy of x, one device -> host copy of (E, g)), so that the reference's own optimiser
(scipy's BFGS in PHF.py:22-24) can drive it unchanged.

``lbfgs`` keeps the whole optimiser state on the device: the iterate, the gradient and m pairs of
(step, gradient change) for the two-loop recursion (Nocedal and Wright, "Numerical Optimization",
Algorithm 7.4), with a backtracking Armijo line search.  Each function evaluation ends with ONE
device -> host read of three numbers (the energy, the directional derivative of the step and the
largest gradient element) that the line search and the stopping test need; nothing else crosses
to the host.  At n = 200 the dense BFGS inverse Hessian of the reference's optimiser would hold
(2 (M - N) N)^2 = 3.6e9 numbers; the limited-memory form keeps m of those vectors.
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Plan, check_status

__all__ = ["DeviceEandG", "lbfgs", "thouless_to_mos"]


def thouless_to_mos(Z: torch.Tensor) -> torch.Tensor:
    """Thouless2MOs (PHFTools.py:280-290) on the device: the orthonormal orbitals (M x M) whose first N
    columns span [I; Z], from the Cholesky factors of I + Z^T Z* and I + Z* Z^T (MLdecompose,
    PHFTools.py:221-228)."""
    V, N = Z.shape
    M = V + N
    eye_n = torch.eye(N, dtype=Z.dtype, device=Z.device)
    eye_v = torch.eye(V, dtype=Z.dtype, device=Z.device)
    mos = torch.eye(M, dtype=Z.dtype, device=Z.device)
    mos[N:, :N] = Z
    mos[:N, N:] = -Z.conj().T
    L = torch.linalg.cholesky(eye_n + Z.T @ Z.conj())
    Mf = torch.linalg.cholesky(eye_v + Z.conj() @ Z.T)
    out = torch.empty_like(mos)
    out[:, :N] = mos[:, :N] @ torch.linalg.inv(L).T
    out[:, N:] = mos[:, N:] @ torch.linalg.inv(Mf).T
    return out


class DeviceEandG:
    """EandG (PHF.py:55-91) on the GPU for one plan.

    ``plan`` is a Plan created with the reference gradient (gradient="reference"); ``basis`` says
    which basis its eval_device takes the determinant in: "ao" for a Cholesky plan (C = Ref [I; z],
    Ref the plan's ``ref``) or "mo" for a dense plan whose HOne/HTwo are already in the Ref-MO basis
    (C = [I; z]).  The projections of PHF.py:58-66 follow the reference's switches: ``nfo`` frozen
    orbitals (FrozenProj, with ``nocc_ao`` occupied spatial orbitals), ``cmplxconj`` (0 drops the
    imaginary part), ``sp`` (2 keeps the Sz-conserving blocks, SzProj), ``is_rhf`` (RHFProj); the
    last three need ``nocc_a`` / ``nvrt_a``, the alpha occupied and virtual counts."""

    def __init__(self, plan: Plan, basis="ao", *, cmplxconj=1, sp=1, is_rhf=False, nfo=0, nocc_ao=None,
                 nocc_a=None, nvrt_a=None, device="cuda"):
        if plan.gradient != "reference":
            raise ValueError("DeviceEandG returns the reference's gradient: create the plan with "
                             "gradient='reference'")
        if basis not in ("ao", "mo"):
            raise ValueError("basis must be 'ao' or 'mo'")
        self.plan, self.basis = plan, basis
        self.M, self.N, self.nci = plan.nso, plan.nocc, plan.nci
        self.ncisp, self.ncipg = plan._g.ncisp, plan._g.ncipg
        self.V = self.M - self.N
        self.dev = torch.device(device)
        self.cmplxconj, self.sp, self.is_rhf, self.nfo = int(cmplxconj), int(sp), bool(is_rhf), int(nfo)
        self.nocc_ao, self.nocc_a, self.nvrt_a = nocc_ao, nocc_a, nvrt_a
        if (self.sp == 2 or self.is_rhf) and (nocc_a is None or nvrt_a is None):
            raise ValueError("SzProj / RHFProj need nocc_a and nvrt_a")
        if self.nfo > 0 and nocc_ao is None:
            raise ValueError("FrozenProj needs nocc_ao")
        self.ref = torch.from_numpy(np.ascontiguousarray(plan.ref)).to(self.dev)
        ns = self.nci * self.nci
        self.out = (torch.empty((ns, 2), dtype=torch.complex128, device=self.dev),
                    torch.empty((ns, self.M, self.N), dtype=torch.complex128, device=self.dev),
                    torch.empty((ns, self.M, self.N), dtype=torch.complex128, device=self.dev))
        self.status = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.evaluations = 0

    # ------------------------------------------------------------------ projections (PHF.py:133-151)
    def project(self, z: torch.Tensor) -> torch.Tensor:
        """FrozenProj, CmplxConj = 0, SzProj and RHFProj in the order of PHF.py:58-66."""
        if self.nfo > 0:
            z = z.clone()
            z[:, :self.nfo] = 0
            z[:, self.nocc_ao:self.nocc_ao + self.nfo] = 0
        if self.cmplxconj == 0:
            z = z.real.to(torch.complex128)
        if self.sp == 2:
            a, v = self.nocc_a, self.nvrt_a
            w = torch.zeros_like(z)
            w[:v, :a] = z[:v, :a]
            w[v:, a:] = z[v:, a:]
            z = w
        if self.is_rhf:
            a, v = self.nocc_a, self.nvrt_a
            w = torch.zeros_like(z)
            w[:v, :a] = z[:v, :a]
            w[v:, a:] = z[:v, :a]
            z = w
        return z

    def _z_of(self, x: torch.Tensor) -> torch.Tensor:
        k = self.V * self.N
        return torch.complex(x[:k], x[k:]).reshape(self.V, self.N)

    def _energy_and_g(self, hs, yg, yr):
        """E0 and sum f*f (Yg - E0 Yr) / sum f*f S (EigenSolver + VecDecomp + LocalG), on the device."""
        nci = self.nci
        if nci == 1:
            H, S = hs[0, 0], hs[0, 1]
            E = H.real / S.real.abs()
            return E, (yg[0] - E * yr[0]) / S
        Hm = hs[:, 0].reshape(nci, nci).T
        Sm = hs[:, 1].reshape(nci, nci).T
        w, U = torch.linalg.eigh(Sm)
        keep = w.abs() > 1e-6                      # the canonical orthogonalisation's threshold (PHFTools.py:7)
        X = U * torch.where(keep, w.abs().clamp_min(1e-300).rsqrt(), torch.zeros_like(w))[None, :]
        h = X.conj().T @ Hm @ X
        # dropped directions get a large diagonal instead of being removed: no data-dependent shapes
        big = 1e6 * (h.abs().max() + 1.0)
        h = h + torch.diag(torch.where(keep, torch.zeros_like(w), big)).to(h.dtype)
        e, V = torch.linalg.eigh(h)
        vec = X @ V[:, 0]
        Mv = vec.reshape(self.ncipg, self.ncisp).T       # VecDecomp's Fortran-order reshape (ncik = 1)
        fpg = Mv[0, :] / Mv[0, 0]
        fsp = Mv[:, 0]
        f = (fsp[:, None] * fpg[None, :]).T.reshape(-1)  # f[m], m = ni + p ncisp
        coef = (f.conj()[:, None] * f[None, :]).T.reshape(-1)  # slot a = m + nci n
        ovlp = (coef * hs[:, 1]).sum()
        E = e[0]
        G = ((coef[:, None, None] * yg).sum(0) - E * (coef[:, None, None] * yr).sum(0)) / ovlp
        return E, G

    def __call__(self, x: torch.Tensor):
        """(E0, g) as device tensors for a device parameter vector x (2 (M - N) N reals); queued on
        the current stream, no host synchronisation.  The evaluation's status words land in
        ``self.status`` (check them with api.check_status after reading them)."""
        z = self.project(self._z_of(x))
        eye = torch.eye(self.N, dtype=torch.complex128, device=self.dev)
        C = torch.cat([eye, z], 0)
        if self.basis == "ao":
            C = self.ref @ C
        C = C.contiguous()
        hs, yg, yr = self.plan.eval_device_async(C, self.out, self.status)
        self.evaluations += 1
        E, G = self._energy_and_g(hs, yg, yr)
        if self.basis == "ao":
            G = self.ref.conj().T @ G
        Gz = self.project(G[self.N:, :])
        g = torch.cat([Gz.real.reshape(-1), Gz.imag.reshape(-1)])
        return E, g

    def host(self, x):
        """EandG with numpy in and out: (float E0, numpy g), as scipy's optimisers call it."""
        xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(self.dev)
        E, g = self(xd)
        out = torch.cat([E.reshape(1).to(torch.float64), g, self.status.to(torch.float64)]).cpu().numpy()
        check_status(out[-2:])
        return float(out[0]), out[1:-2].copy()


def lbfgs(fun, x0, maxiter=100, m=10, gtol=1e-4, c1=1e-4, max_backtrack=30, callback=None):
    """Minimise E(x) with the optimiser state on the device (two-loop L-BFGS, Armijo backtracking).

    ``fun(x)`` returns (E, g) as device tensors without synchronising (DeviceEandG does); ``x0`` is a
    device tensor.  Each function evaluation is followed by one device -> host read of three numbers.
    Stops when the largest gradient element is below ``gtol`` (PHF.py:20 uses 1e-4).  Returns a dict
    with x, E, g (device), the iteration and evaluation counts and the number of host reads."""
    x = x0.clone()
    status = getattr(fun, "status", None)
    pinned = torch.empty(5, dtype=torch.float64, pin_memory=True)
    reads = 0

    def read(*scalars):
        nonlocal reads
        vals = [s.reshape(1).to(torch.float64) for s in scalars]
        if status is not None:
            vals.append(status.to(torch.float64))
        buf = torch.cat(vals)
        pinned[:buf.numel()].copy_(buf, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        reads += 1
        out = pinned[:buf.numel()].numpy().copy()
        if status is not None:
            check_status(out[-2:])
        return out

    E, g = fun(x)
    e_now, gmax = read(E, g.abs().max())[:2]
    S, Y, R = [], [], []           # history on the device: steps, gradient changes, 1 / (y.s)
    it = 0
    trace = [float(e_now)]
    while it < maxiter and gmax > gtol:
        # two-loop recursion: d = -H g
        q = g.clone()
        alphas = []
        for s, y, r in zip(reversed(S), reversed(Y), reversed(R)):
            a = r * torch.dot(s, q)
            alphas.append(a)
            q = q - a * y
        if S:
            gamma = torch.dot(S[-1], Y[-1]) / torch.dot(Y[-1], Y[-1]).clamp_min(1e-300)
            q = gamma * q
        else:
            q = q * min(1.0, 1.0 / max(gmax, 1e-300))
        for (s, y, r), a in zip(zip(S, Y, R), reversed(alphas)):
            b = r * torch.dot(y, q)
            q = q + (a - b) * s
        d = -q
        gd = torch.dot(g, d)
        t = 1.0
        accepted = False
        for _ in range(max_backtrack):
            xn = x + t * d
            En, gn = fun(xn)
            gd_h, e_new, gmax_new = read(gd, En, gn.abs().max())[:3]
            if gd_h >= 0:  # not a descent direction: restart from steepest descent
                S.clear(), Y.clear(), R.clear()
                d = -g * min(1.0, 1.0 / max(gmax, 1e-300))
                gd = torch.dot(g, d)
                t = 1.0
                continue
            if e_new <= e_now + c1 * t * gd_h:
                accepted = True
                break
            t *= 0.5
        if not accepted:
            break
        s = xn - x
        y = gn - g
        ys = torch.dot(y, s)
        # pairs without positive curvature get weight zero (no host decision needed)
        r = torch.where(ys > 1e-30, 1.0 / ys.clamp_min(1e-300), torch.zeros_like(ys))
        S.append(s), Y.append(y), R.append(r)
        if len(S) > m:
            S.pop(0), Y.pop(0), R.pop(0)
        x, g, e_now, gmax = xn, gn, e_new, gmax_new
        it += 1
        trace.append(float(e_now))
        if callback is not None:
            callback(it, e_now, gmax)
    return {"x": x, "E": e_now, "g": g, "gmax": gmax, "iterations": it, "host_reads": reads,
            "evaluations": getattr(fun, "evaluations", None), "energies": trace}
