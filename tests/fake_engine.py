"""CPU stand-in for the native Engine -- TEST INFRASTRUCTURE ONLY.

Implements the Engine method surface (renormalizer_b200._native.Engine) with
torch CPU ops so that the host logic of the sweep engine (QN bookkeeping,
truncation and selection order, sweep control flow, Krylov control flow) can
be exercised in CI without a GPU.  It is installed only by the
``cpu_engine`` fixture; the product never falls back to it -- without the
fixture every call goes to libreno_b200.so and fails loudly without a GPU.
"""
import torch


def _chk(*ts):
    """the native engine reads raw memory: lazy conj/neg views must be resolved first"""
    for t in ts:
        if isinstance(t, torch.Tensor):
            assert not (t.is_conj() or t.is_neg()), "lazy conj/neg view passed to the engine"


class FakeEngine:
    def __init__(self):
        self.launches = 0

    def __getattribute__(self, name):
        attr = object.__getattribute__(self, name)
        if name in ("heff_apply", "heff_apply_grouped", "heff_backward", "heff_diag", "env_update", "vec_norm", "vec_dotc", "krylov_alpha", "krylov_orth",
                    "scale_inv", "lincomb", "allclose", "axpy", "precond", "qn_gather"):
            def checked(*a, **k):
                _chk(*a)
                return attr(*a, **k)
            return checked
        return attr

    def sync_stream(self):
        pass

    # ------------------------------------------------------------ contractions
    def heff_apply(self, d, L, W1, W2, R, psi, y):
        if d.nsite == 0:
            r = torch.einsum("abc,lbk,ck->al", L.to(y.dtype), R.to(y.dtype), psi.to(y.dtype))
        elif d.nsite == 1:
            r = torch.einsum("abc,bdef,lfk,cek->adl", L.to(y.dtype), W1.to(y.dtype), R.to(y.dtype), psi.to(y.dtype))
        else:
            # pairwise, in the reference's contraction order (a single 5-operand
            # einsum would build an M^2 d^2 w^2-sized intermediate)
            t = torch.einsum("abc,cehk->abehk", L.to(y.dtype), psi.to(y.dtype))
            t = torch.einsum("abehk,bdef->adfhk", t, W1.to(y.dtype))
            t = torch.einsum("adfhk,fghj->adgjk", t, W2.to(y.dtype))
            r = torch.einsum("adgjk,ljk->adgl", t, R.to(y.dtype))
        y.copy_(r)

    def heff_apply_grouped(self, descs, Ls, W1s, W2s, Rs, psis, ys):
        for d, L, W1, W2, R, psi, y in zip(descs, Ls, W1s, W2s, Rs, psis, ys):
            self.heff_apply(d, L, W1, W2, R, psi, y)

    def heff_backward(self, d, L, W1, W2, R, psi, gy, gpsi, gL, gW1, gW2, gR):
        spec = {0: "abc,lbk,ck->al", 1: "abc,bdef,lfk,cek->adl", 2: "abc,bdef,fghj,ljk,cehk->adgl"}[d.nsite]
        dt = gy.dtype
        leaves = [t.detach().to(dt).requires_grad_(True) for t in [L] + [w for w in (W1, W2) if w is not None] +
                  [R, psi]]
        with torch.enable_grad():
            y = torch.einsum(spec, *leaves)
            grads = torch.autograd.grad(y, leaves, gy)
        outs = [gL] + [o for o, w in ((gW1, W1), (gW2, W2)) if w is not None] + [gR, gpsi]
        for o, g in zip(outs, grads):
            if o is not None:
                o.copy_(g)

    def heff_diag(self, d, L, W1, W2, R, out):
        tl = torch.einsum("aba->ba", L).real
        tr = torch.einsum("aba->ba", R).real
        t0 = torch.einsum("abbc->abc", W1).real
        if d.nsite == 1:
            out.copy_(torch.einsum("ba,bcg,gf->acf", tl, t0, tr))
        else:
            t1 = torch.einsum("abbc->abc", W2).real
            out.copy_(torch.einsum("ba,bce,edg,gf->acdf", tl, t0, t1, tr))

    def env_update(self, d, E, W, ket, bra, out):
        dt = out.dtype
        b = bra.to(dt) if bra is not None else ket.to(dt).conj()
        if d.side == 0:
            r = torch.einsum("abc,adf,bdeg,ceh->fgh", E.to(dt), b, W.to(dt), ket.to(dt))
        else:
            r = torch.einsum("fda,abc,gdeb,hec->fgh", b, E.to(dt), W.to(dt), ket.to(dt))
        out.copy_(r)

    def matmul(self, A, B, conj_a=False, conj_b=False, prec="fp64"):
        dt = torch.complex128 if (A.is_complex() or B.is_complex()) else torch.float64
        a, b = A.to(dt), B.to(dt)
        if conj_a:
            a = a.conj()
        if conj_b:
            b = b.conj()
        return (a @ b).resolve_conj().contiguous()

    def qr_blocks(self, mats):
        out = [torch.linalg.qr(a, mode="reduced") for a in mats]
        return [q.contiguous() for q, _ in out], [r.contiguous() for _, r in out]

    # ------------------------------------------------------------ vectors
    def vec_norm(self, x, out):
        out[0] = torch.linalg.vector_norm(x)

    def vec_dotc(self, x, y, out):
        v = torch.vdot(x.reshape(-1).to(torch.complex128), y.reshape(-1).to(torch.complex128))
        out[0], out[1] = v.real, v.imag

    def krylov_alpha(self, w, v, ab, j):
        ab[2 * j] = torch.vdot(w.reshape(-1), v.reshape(-1)).real

    def krylov_orth(self, w, v, vprev, ab, j):
        t = ab[2 * j] * v
        if j > 0:
            t = t + ab[2 * j - 1] * vprev
        w -= t
        ab[2 * j + 1] = torch.linalg.vector_norm(w)

    def scale_inv(self, x, s, out):
        out.copy_(x / s[0])

    def lincomb(self, V, k, coef, out):
        c = torch.complex(coef[0:2 * k:2], coef[1:2 * k:2])
        if V.is_complex():
            out.copy_(c @ V[:k])
        else:
            out.copy_(c.real @ V[:k])

    def allclose(self, a, b, rtol, atol, flag):
        flag[0] = 1.0 if bool(torch.all(torch.abs(a - b) <= atol + rtol * torch.abs(b))) else 0.0

    def vec_grouped(self, op, items, rtol=0.0, atol=0.0):
        """reno_vec_grouped: the single operation on every item, in order"""
        for n, dt, j, x, y, out, sc, s, ldv in items:
            _chk(x, y, out, sc, s)
            if op == 0:
                self.vec_norm(x, sc)
            elif op == 1:
                self.krylov_alpha(x, y, sc, j)
            elif op == 2:
                self.krylov_orth(out, x, y, sc, j)
            elif op == 3:
                self.scale_inv(x, s, out)
            elif op == 4:
                self.lincomb(x, j, s, out)
            else:
                self.allclose(x, y, rtol, atol, sc)

    def axpy(self, y, x, c, sign=1.0):
        cc = complex(c[0].item(), c[1].item() if y.is_complex() else 0.0) * sign
        y += (cc if y.is_complex() else cc.real) * x

    def precond(self, r, hdiag, e, shift, out):
        out.copy_(r / (hdiag - e[0] + shift))

    # ------------------------------------------------------------ QN movers
    def qn_gather(self, mat, rows, cols, out):
        out.copy_(mat[rows][:, cols])

    def qn_scatter(self, src, rows, scols, dcols, sigma, dst, dst_rs, dst_cs):
        vals = src[:, scols].to(dst.dtype)
        if sigma is not None:
            vals = vals * sigma.to(vals.real.dtype)
        idx = rows[:, None] * dst_rs + dcols[None, :] * dst_cs
        dst.view(-1)[idx.reshape(-1)] = vals.reshape(-1)
