"""Learned extrapolator of the long-time tail of the TBPM DOS correlation C(t).

A short propagation gives C(t) for t = 0..n_in; the network predicts
C(n_in+1 .. n_in+n_out) (real and imaginary parts), so that the DOS can be
evaluated at the resolution of the full length without propagating it.  The
full-length plain propagation remains the fallback and the yardstick:
`evaluate` compares the DOS of (short propagation + predicted tail) with the
DOS of the full propagation.

Network (all dense/convolution products are the BF16 tensor-core GEMM of
libtbpm_b200 with FP32 accumulation; activations channel-last):

    input  (n_in, 2)  -> channels padded to 8
    conv1d 8   -> 256, kernel 5, stride 2, GELU      (n_in/2 positions)
    conv1d 256 -> 256, kernel 5, stride 2, GELU      (n_in/4)
    conv1d 256 -> 256, kernel 5, stride 4, GELU      (n_in/16)
    dense  (n_in/16 * 256) -> 2*n_out                 (the fourth layer: a
           convolution whose kernel spans the whole remaining sequence)

Training: mean-squared error on the scaled tail, AdamW on FP32 master
weights with BF16 working copies, forward and backward entirely in the
library's kernels; torch only holds the device buffers and the stream.
"""

import math
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _native as nat


class TailNet:
    """BF16 convolutional tail extrapolator trained by libtbpm_b200 kernels."""

    def __init__(self, n_in: int = 256, n_out: int = 1792, width: int = 256, kernel: int = 5,
                 strides=(2, 2, 4), c_in: int = 8, device: int = 0, seed: int = 0) -> None:
        import torch
        self.torch = torch
        self.lib = nat.load_library()
        self.dev = torch.device("cuda", device)
        self.n_in, self.n_out, self.width, self.kernel = n_in, n_out, width, kernel
        self.c_in = c_in
        pad = kernel // 2
        self.convs: List[Dict] = []
        L, C = n_in, c_in
        for s in strides:
            Lout = (L + 2 * pad - kernel) // s + 1
            self.convs.append({"L": L, "C": C, "Lout": Lout, "Cout": width, "s": s, "p": pad})
            L, C = Lout, width
        self.F = L * C
        self.O = 2 * n_out
        rng = np.random.default_rng(seed)
        self.params: List[Dict] = []
        for cv in self.convs:
            fan_in = kernel * cv["C"]
            w = rng.standard_normal((cv["Cout"], fan_in)) * math.sqrt(2.0 / fan_in)
            if cv is self.convs[0]:
                w.reshape(cv["Cout"], kernel, cv["C"])[:, :, 2:] = 0.0  # padded channels
            self._add_param(w)
            self._add_param(np.zeros(cv["Cout"]))
        self._add_param(rng.standard_normal((self.O, self.F)) * math.sqrt(1.0 / self.F) * 0.1)
        self._add_param(np.zeros(self.O))
        self.step = 0
        self.in_scale = 1.0
        self.out_scale = 1.0
        self._work = torch.zeros(256, dtype=torch.float64, device=self.dev)
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.dev)

    # -- parameters ------------------------------------------------------------
    def _add_param(self, w: np.ndarray) -> None:
        t = self.torch
        p = {"w": t.tensor(np.asarray(w, dtype=np.float32), device=self.dev)}
        p["g"] = t.zeros_like(p["w"])
        p["m"] = t.zeros_like(p["w"])
        p["v"] = t.zeros_like(p["w"])
        p["bf"] = t.zeros(p["w"].shape, dtype=t.bfloat16, device=self.dev)
        self.params.append(p)
        self._cast(p)

    def _cast(self, p) -> None:
        self._chk(self.lib.tbpm_nn_cast_bf16(p["w"].data_ptr(), p["w"].numel(),
                                             p["bf"].data_ptr(), self._stream()))

    def _stream(self) -> int:
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    @staticmethod
    def _chk(rc: int) -> None:
        if rc != nat.TBPM_OK:
            raise nat.TbpmError(rc, f"libtbpm_b200 nn kernel failed with status {rc}")

    def state_dict(self) -> Dict[str, np.ndarray]:
        d = {f"p{i}": p["w"].cpu().numpy() for i, p in enumerate(self.params)}
        d["in_scale"] = np.array(self.in_scale)
        d["out_scale"] = np.array(self.out_scale)
        return d

    def load_state_dict(self, d: Dict[str, np.ndarray]) -> None:
        for i, p in enumerate(self.params):
            p["w"].copy_(self.torch.tensor(d[f"p{i}"], device=self.dev))
            self._cast(p)
        self.in_scale = float(d["in_scale"])
        self.out_scale = float(d["out_scale"])

    # -- building blocks ---------------------------------------------------------
    def _gemm(self, A, lda, B, ldb, C, M, N, K, beta=0.0) -> None:
        self._chk(self.lib.tbpm_nn_gemm_tn(A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), N,
                                           M, N, K, 1.0, beta, self._stream()))

    def _transpose(self, x, rows, cols):
        out = self.torch.empty((cols, rows), dtype=self.torch.bfloat16, device=self.dev)
        self._chk(self.lib.tbpm_nn_transpose_bf16(x.data_ptr(), rows, cols, out.data_ptr(),
                                                  self._stream()))
        return out

    def _pack_input(self, x: np.ndarray):
        """(B, n_in, 2) float -> channel-padded BF16 (B, n_in, c_in) on the device."""
        t = self.torch
        B = x.shape[0]
        xp = np.zeros((B, self.n_in, self.c_in), dtype=np.float32)
        xp[:, :, :2] = x * self.in_scale
        return t.tensor(xp, device=self.dev).to(t.bfloat16)

    # -- forward / backward ------------------------------------------------------
    def forward(self, x: np.ndarray, keep: bool = False):
        """x: (B, n_in, 2) real/imaginary parts of C(1..n_in).  Returns the
        scaled prediction (B, 2*n_out) as a device FP32 tensor."""
        t = self.torch
        B = x.shape[0]
        if B % 8:
            raise ValueError("batch size must be a multiple of 8")
        a = self._pack_input(x)
        cache = []
        for li, cv in enumerate(self.convs):
            W, b = self.params[2 * li], self.params[2 * li + 1]
            K = self.kernel * cv["C"]
            rows = B * cv["Lout"]
            xcol = t.empty((rows, K), dtype=t.bfloat16, device=self.dev)
            self._chk(self.lib.tbpm_nn_im2col(a.data_ptr(), B, cv["L"], cv["C"], self.kernel,
                                              cv["s"], cv["p"], cv["Lout"], xcol.data_ptr(),
                                              self._stream()))
            z = t.empty((rows, cv["Cout"]), dtype=t.float32, device=self.dev)
            self._gemm(xcol, K, W["bf"], K, z, rows, cv["Cout"], K)
            pre = t.empty_like(z)
            a = t.empty((rows, cv["Cout"]), dtype=t.bfloat16, device=self.dev)
            self._chk(self.lib.tbpm_nn_bias_act(z.data_ptr(), b["w"].data_ptr(), rows, cv["Cout"],
                                                1, pre.data_ptr(), a.data_ptr(), None,
                                                self._stream()))
            cache.append((xcol, pre))
        Wd, bd = self.params[-2], self.params[-1]
        h = a.view(B, self.F)
        zd = t.empty((B, self.O), dtype=t.float32, device=self.dev)
        self._gemm(h, self.F, Wd["bf"], self.F, zd, B, self.O, self.F)
        out = t.empty_like(zd)
        self._chk(self.lib.tbpm_nn_bias_act(zd.data_ptr(), bd["w"].data_ptr(), B, self.O, 0, None,
                                            None, out.data_ptr(), self._stream()))
        if keep:
            self._cache = (B, cache, h)
        return out

    def backward(self, grad_out) -> None:
        """Gradients of all parameters from d(loss)/d(output) (B, 2*n_out)."""
        t = self.torch
        B, cache, h = self._cache
        Wd, bd = self.params[-2], self.params[-1]
        g_bf = grad_out.to(t.bfloat16)
        gT = self._transpose(g_bf, B, self.O)
        hT = self._transpose(h, B, self.F)
        self._gemm(gT, B, hT, B, Wd["g"], self.O, self.F, B)
        self._chk(self.lib.tbpm_nn_colsum(grad_out.data_ptr(), B, self.O, bd["g"].data_ptr(),
                                          self._stream()))
        wdT = self._transpose(Wd["bf"], self.O, self.F)
        dA = t.empty((B, self.F), dtype=t.float32, device=self.dev)
        self._gemm(g_bf, self.O, wdT, self.O, dA, B, self.F, self.O)
        for li in range(len(self.convs) - 1, -1, -1):
            cv = self.convs[li]
            W, b = self.params[2 * li], self.params[2 * li + 1]
            xcol, pre = cache[li]
            rows = B * cv["Lout"]
            K = self.kernel * cv["C"]
            dz = t.empty((rows, cv["Cout"]), dtype=t.float32, device=self.dev)
            dzb = t.empty((rows, cv["Cout"]), dtype=t.bfloat16, device=self.dev)
            self._chk(self.lib.tbpm_nn_act_backward(dA.data_ptr(), pre.data_ptr(), dz.numel(), 1,
                                                    dz.data_ptr(), dzb.data_ptr(),
                                                    self._stream()))
            self._chk(self.lib.tbpm_nn_colsum(dz.data_ptr(), rows, cv["Cout"], b["g"].data_ptr(),
                                              self._stream()))
            dzT = self._transpose(dzb, rows, cv["Cout"])
            xcolT = self._transpose(xcol, rows, K)
            self._gemm(dzT, rows, xcolT, rows, W["g"], cv["Cout"], K, rows)
            if li > 0:
                wT = self._transpose(W["bf"], cv["Cout"], K)
                dxcol = t.empty((rows, K), dtype=t.float32, device=self.dev)
                self._gemm(dzb, cv["Cout"], wT, cv["Cout"], dxcol, rows, K, cv["Cout"])
                dA = t.empty((B * cv["L"], cv["C"]), dtype=t.float32, device=self.dev)
                self._chk(self.lib.tbpm_nn_col2im(dxcol.data_ptr(), B, cv["L"], cv["C"],
                                                  self.kernel, cv["s"], cv["p"], cv["Lout"],
                                                  dA.data_ptr(), self._stream()))

    def loss_and_grad(self, pred, target):
        t = self.torch
        grad = t.empty_like(pred)
        self._chk(self.lib.tbpm_nn_mse(pred.data_ptr(), target.data_ptr(), pred.numel(),
                                       grad.data_ptr(), self._work.data_ptr(),
                                       self._loss.data_ptr(), self._stream()))
        return self._loss, grad

    def adam_step(self, lr: float, weight_decay: float = 1e-4, b1: float = 0.9,
                  b2: float = 0.999, eps: float = 1e-8) -> None:
        self.step += 1
        for p in self.params:
            self._chk(self.lib.tbpm_nn_adam(p["w"].data_ptr(), p["g"].data_ptr(),
                                            p["m"].data_ptr(), p["v"].data_ptr(), p["w"].numel(),
                                            lr, b1, b2, eps, weight_decay, self.step,
                                            p["bf"].data_ptr(), self._stream()))

    # -- data scaling, training, inference ------------------------------------------
    def fit_scales(self, x: np.ndarray, y: np.ndarray) -> None:
        self.in_scale = 1.0 / max(float(np.sqrt(np.mean(x ** 2))), 1e-12)
        self.out_scale = 1.0 / max(float(np.sqrt(np.mean(y ** 2))), 1e-12)

    def _snapshot(self):
        return [p["w"].clone() for p in self.params]

    def _restore(self, snap) -> None:
        for p, w in zip(self.params, snap):
            p["w"].copy_(w)
            self._cast(p)

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int = 100, batch: int = 64,
              lr: float = 1e-3, weight_decay: float = 1e-4, seed: int = 0,
              x_val: Optional[np.ndarray] = None, y_val: Optional[np.ndarray] = None,
              patience: Optional[int] = None, log=None) -> Dict[str, list]:
        """x: (n, n_in, 2), y: (n, n_out, 2).  Cosine-decayed AdamW.  With a
        validation set the weights of the best validation epoch are kept
        (early stopping after `patience` epochs without improvement)."""
        t = self.torch
        n = x.shape[0]
        batch = max(8, (min(batch, n) // 8) * 8)
        ys = (y.reshape(n, -1) * self.out_scale).astype(np.float32)
        rng = np.random.default_rng(seed)
        hist = {"train": [], "val": [], "best_epoch": -1}
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        it = 0
        best, best_snap, since = math.inf, None, 0
        if x_val is not None:
            best = self.mse(x_val, y_val)
            best_snap = self._snapshot()
            hist["val_initial"] = best
        for ep in range(epochs):
            perm = rng.permutation(n)
            acc = 0.0
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                pred = self.forward(x[idx], keep=True)
                target = t.tensor(ys[idx], device=self.dev)
                loss, grad = self.loss_and_grad(pred, target)
                self.backward(grad)
                cur = lr * 0.5 * (1 + math.cos(math.pi * it / total))
                self.adam_step(cur, weight_decay)
                acc += float(loss.item())
                it += 1
            hist["train"].append(acc / steps_per_epoch)
            if x_val is not None:
                v = self.mse(x_val, y_val)
                hist["val"].append(v)
                if v < best:
                    best, best_snap, since = v, self._snapshot(), 0
                    hist["best_epoch"] = ep
                else:
                    since += 1
            if log and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                log(f"epoch {ep}: train {hist['train'][-1]:.4e}"
                    + (f" val {hist['val'][-1]:.4e}" if hist["val"] else ""))
            if patience is not None and x_val is not None and since > patience:
                break
        if best_snap is not None:
            self._restore(best_snap)
            hist["val_best"] = best
        return hist

    def predict(self, x: np.ndarray) -> np.ndarray:
        """(B, n_in, 2) -> predicted tail (B, n_out, 2) in the units of C(t)."""
        B = x.shape[0]
        pad = (-B) % 8
        xp = np.concatenate([x, np.zeros((pad,) + x.shape[1:], dtype=x.dtype)]) if pad else x
        out = self.forward(xp).cpu().numpy()[:B]
        return (out / self.out_scale).reshape(B, self.n_out, 2)

    def mse(self, x: np.ndarray, y: np.ndarray) -> float:
        p = self.predict(x)
        return float(np.mean(((p - y) * self.out_scale) ** 2))


# ---- data and evaluation ----------------------------------------------------------

def curves_to_xy(corr: np.ndarray, n_in: int, n_out: int) -> Tuple[np.ndarray, np.ndarray]:
    """corr (n, >= n_in+n_out+1) complex -> x (n, n_in, 2) for t = 1..n_in and
    y (n, n_out, 2) for t = n_in+1..n_in+n_out."""
    c = np.asarray(corr)
    x = np.stack([c[:, 1:n_in + 1].real, c[:, 1:n_in + 1].imag], axis=-1)
    y = np.stack([c[:, n_in + 1:n_in + n_out + 1].real, c[:, n_in + 1:n_in + n_out + 1].imag],
                 axis=-1)
    return x.astype(np.float32), y.astype(np.float32)


def extend(corr_short: np.ndarray, tail: np.ndarray) -> np.ndarray:
    """C(0..n_in) followed by the predicted C(n_in+1..n_in+n_out)."""
    return np.concatenate([corr_short, tail[..., 0] + 1j * tail[..., 1]], axis=-1)


def dos_from_corr(corr: np.ndarray, energy_range: float) -> Tuple[np.ndarray, np.ndarray]:
    """Analyzer.calc_dos (Hanning window, tnr = len(corr) - 1)."""
    from .tbpm import Analyzer, Config

    class _S:
        pass

    s = _S()
    s.energy_range = energy_range
    cfg = Config()
    cfg.generic["nr_time_steps"] = len(corr) - 1
    return Analyzer(s, cfg, dimension=2).calc_dos(corr)


def dos_l1(corr: np.ndarray, corr_ref: np.ndarray, energy_range: float) -> float:
    """L1 distance of the DOS of corr and of corr_ref on the grid of corr_ref;
    a shorter corr is evaluated at its own resolution and interpolated."""
    e_ref, d_ref = dos_from_corr(corr_ref, energy_range)
    e, d = dos_from_corr(corr, energy_range)
    if len(corr) != len(corr_ref):
        d = np.interp(e_ref, e, d)
        d /= np.sum(d) * (e_ref[1] - e_ref[0])
    return float(np.sum(np.abs(d - d_ref)) * (e_ref[1] - e_ref[0]))


def time_gemm(m: int, n: int, k: int, reps: int = 10, warmup: int = 3) -> Dict[str, float]:
    """Time the network's tensor-core GEMM (tbpm_nn_gemm_tn, tcgen05) and the
    mma.sync GEMM on random BF16 operands of shape (m, k) x (n, k)^T with CUDA
    events; returns milliseconds and TF/s of each."""
    import torch
    lib = nat.load_library()
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda").to(torch.bfloat16)
    c = torch.zeros(m, n, device="cuda")
    out: Dict[str, float] = {"m": m, "n": n, "k": k}
    for name, fn in (("tcgen05", lib.tbpm_nn_gemm_tn), ("mma_sync", lib.tbpm_nn_gemm_tn_mma)):
        for _ in range(warmup):
            fn(a.data_ptr(), k, b.data_ptr(), k, c.data_ptr(), n, m, n, k, 1.0, 0.0, s)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn(a.data_ptr(), k, b.data_ptr(), k, c.data_ptr(), n, m, n, k, 1.0, 0.0, s)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(reps, 1)
        out[name + "_ms"] = ms
        out[name + "_tflops"] = 2.0 * m * n * k / ms / 1e9
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time the tail network's GEMM kernels")
    ap.add_argument("--shape", type=int, nargs=3, default=[4096, 4096, 4096],
                    metavar=("M", "N", "K"))
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    print(json.dumps(time_gemm(*args.shape, reps=args.reps, warmup=args.warmup)))
