"""Learned proposal (MADE) and rejection sampling against the engine's p(x).

* ``MadeProposal``: masked autoregressive network (inputs in scan order, two hidden
  layers) trained on the device by the library's BF16 kernels (``rgs_mlp_fwd/bwd/adam``)
  on exact samples and the exact conditionals p(x_v = 1 | prefix) that the chain-rule
  sampler returns (soft-target cross entropy).
* ``rejection_sample``: the reference's accept rule, accept iff u < min(1, p / (c q))
  (``W/rejection_sampler.py:18-23``): with the uniform proposal q = 2^-n and c = cap it IS
  the reference's capped rule; with a learned q it is rejection sampling, Born-exact
  exactly when p <= c q for every x.  Decisions whose uniform lies within ``margin`` of
  the acceptance probability are re-decided with the FP64 (complex128) scan
  (``W/audit_all_proposals_fp64.py:36-54``).
* ``calibrate_envelope``: c from held-out exact samples, with the deficit mass
  D = E_{x~p}[max(0, 1 - c q / p)] (the total-variation distance of the output from p)
  estimated on the same samples.
"""
import ctypes
import math
import time

import numpy as np
import torch

from . import _lib

__all__ = ["made_masks", "MadeProposal", "rejection_sample", "calibrate_envelope", "capped_rejection"]


def made_masks(n, hidden):
    """MADE connectivity for inputs ordered 1..n (Germain et al. 2015): hidden unit k has
    degree 1 + (k mod (n - 1)); output d sees hidden units of degree < d."""
    deg_in = np.arange(1, n + 1)
    deg_h = (np.arange(hidden) % max(1, n - 1)) + 1
    m1 = (deg_h[:, None] >= deg_in[None, :]).astype(np.uint8)          # [hidden][n]
    m2 = (deg_h[:, None] >= deg_h[None, :]).astype(np.uint8)           # [hidden][hidden]
    m3 = (deg_in[:, None] > deg_h[None, :]).astype(np.uint8)           # [n][hidden]
    return m1, m2, m3


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class MadeProposal:
    """q(x) = prod_d q(x_d | x_<d) over bits in scan order."""

    def __init__(self, n, hidden=512, device=0, seed=0):
        self.n, self.hidden = int(n), int(hidden)
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        rng = np.random.default_rng(seed)
        masks = made_masks(self.n, self.hidden)
        shapes = [(self.hidden, self.n), (self.hidden, self.hidden), (self.n, self.hidden)]
        self.masks = [torch.from_numpy(m).to(self.device) for m in masks]
        self.w, self.b = [], []
        for (o, i), m in zip(shapes, masks):
            w = rng.normal(0.0, math.sqrt(2.0 / max(1, m.sum(axis=1).mean())), size=(o, i)) * m
            self.w.append(torch.from_numpy(w.astype(np.float32)).to(self.device))
            self.b.append(torch.zeros(o, dtype=torch.float32, device=self.device))
        self.wb = [(w * m).to(torch.bfloat16) for w, m in zip(self.w, self.masks)]
        self.opt = [(torch.zeros_like(t), torch.zeros_like(t)) for t in self.w + self.b]
        self.t = 0
        self._bufs = {}

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _buffers(self, batch):
        if batch not in self._bufs:
            d, h, n = self.device, self.hidden, self.n
            bf = dict(dtype=torch.bfloat16, device=d)
            self._bufs[batch] = dict(
                x=torch.zeros((batch, n), **bf), h1=torch.empty((batch, h), **bf), h2=torch.empty((batch, h), **bf),
                z=torch.empty((batch, n), dtype=torch.float32, device=d), dz=torch.empty((batch, n), **bf),
                dh2=torch.empty((batch, h), **bf), dh1=torch.empty((batch, h), **bf),
                logq=torch.empty(batch, dtype=torch.float64, device=d),
                loss=torch.empty(256, dtype=torch.float64, device=d))
        return self._bufs[batch]

    def _wargs(self):
        w1, w2, w3 = self.wb
        b1, b2, b3 = self.b
        return [_p(w1), _p(b1), _p(w2), _p(b2), _p(w3), _p(b3)]

    # ------------------------------------------------------------------ device ops
    def _input(self, x):
        """Row-major bf16 [batch, n] on this device (the kernels read raw row-major memory)."""
        if x.dim() != 2 or x.shape[1] != self.n:
            raise ValueError(f"inputs must have shape (batch, {self.n})")
        return x.to(device=self.device, dtype=torch.bfloat16).contiguous()

    def forward(self, x_bf16):
        """Logits z [batch, n] for bf16 inputs on the device."""
        x_bf16 = self._input(x_bf16)
        batch = int(x_bf16.shape[0])
        buf = self._buffers(batch)
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_mlp_fwd(batch, self.n, self.hidden, _p(x_bf16), *self._wargs(),
                                              _p(buf["h1"]), _p(buf["h2"]), _p(buf["z"]), self._stream()))
        return buf["z"]

    def gradients(self, x_bf16, target):
        """(loss, [gW1, gb1, gW2, gb2, gW3, gb3]) for one batch; target = exact conditionals."""
        x_bf16 = self._input(x_bf16)
        target = target.to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(target.shape) != tuple(x_bf16.shape):
            raise ValueError("targets must match the inputs' shape")
        batch = int(x_bf16.shape[0])
        buf = self._buffers(batch)
        self.forward(x_bf16)
        g = [torch.empty_like(t) for t in (self.w[0], self.b[0], self.w[1], self.b[1], self.w[2], self.b[2])]
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_mlp_bwd(
                batch, self.n, self.hidden, _p(x_bf16), _p(self.wb[1]), _p(self.wb[2]), _p(buf["h1"]),
                _p(buf["h2"]), _p(buf["z"]), _p(target), _p(self.masks[0]), _p(self.masks[1]), _p(self.masks[2]),
                _p(buf["dz"]), _p(buf["dh2"]), _p(buf["dh1"]), *[_p(t) for t in g], _p(buf["loss"]), 256,
                self._stream()))
        loss = float(buf["loss"].sum().item()) / batch
        return loss, g

    def train_batch(self, x_bf16, target, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        loss, g = self.gradients(x_bf16, target)
        self.t += 1
        params = [(self.w[0], g[0], self.masks[0], self.wb[0]), (self.b[0], g[1], None, None),
                  (self.w[1], g[2], self.masks[1], self.wb[1]), (self.b[1], g[3], None, None),
                  (self.w[2], g[4], self.masks[2], self.wb[2]), (self.b[2], g[5], None, None)]
        states = [self.opt[0], self.opt[3], self.opt[1], self.opt[4], self.opt[2], self.opt[5]]
        with torch.cuda.device(self.device):
            for (w, gr, m, wb), (s1, s2) in zip(params, states):
                _lib.check(_lib.lib().rgs_mlp_adam(_p(w), _p(gr), _p(s1), _p(s2), _p(m), _p(wb), w.numel(), lr,
                                                   beta1, beta2, eps, self.t, self._stream()))
        return loss

    def fit(self, bits_scan, cond, epochs=4, batch=4096, lr=2e-3, seed=0):
        """Train on exact samples (bits in scan order) and their exact conditionals."""
        x_all = torch.as_tensor(np.ascontiguousarray(bits_scan, dtype=np.float32)).to(self.device).to(torch.bfloat16)
        c_all = torch.as_tensor(np.ascontiguousarray(cond, dtype=np.float32)).to(self.device)
        rng = np.random.default_rng(seed)
        losses = []
        count = len(x_all) - len(x_all) % batch
        for _ in range(epochs):
            perm = torch.as_tensor(rng.permutation(len(x_all))[:count], device=self.device)
            for s in range(0, count, batch):
                idx = perm[s:s + batch]
                losses.append(self.train_batch(x_all[idx].contiguous(), c_all[idx].contiguous(), lr=lr))
        return losses

    def sample(self, count, seed=0, first=0):
        """(bits bf16 [count, n] on device, log q float64 [count] on device)."""
        buf = self._buffers(count)
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_mlp_sample(count, self.n, self.hidden, *self._wargs(), int(seed), int(first),
                                                 _p(buf["x"]), _p(buf["logq"]), _p(buf["h1"]), _p(buf["h2"]),
                                                 _p(buf["z"]), self._stream()))
        return buf["x"], buf["logq"]

    def sample_mixture(self, count, mix, seed=0, first=0):
        """Samples of the defensive mixture q_mix = (1 - mix) q + mix 2^-n with log q_mix:
        each row of a network sample is replaced, with probability `mix`, by uniform bits
        (seeded host draws), and log q_mix of every row comes from one log-q pass.  Where
        the network underestimates p, q_mix >= mix 2^-n bounds p / q_mix by 2^n p / mix,
        so the exact envelope max p / q_mix stays near the bulk's ratio."""
        if not 0.0 < mix < 1.0:
            raise ValueError("mix must lie in (0, 1)")
        x, _ = self.sample(count, seed, first)
        rng = np.random.default_rng([int(seed) & (2 ** 63 - 1), int(first) & (2 ** 63 - 1), 0x6D6978])
        repl = rng.random(count) < mix
        if repl.any():
            u = torch.from_numpy(rng.integers(0, 2, (int(repl.sum()), self.n)).astype(np.float32)).to(self.device)
            idx = torch.from_numpy(np.flatnonzero(repl)).to(self.device)
            x = x.clone()
            x[idx] = u.to(torch.bfloat16)
        lq = self.log_q(x)
        return x, self.mixture_log_q(lq, mix)

    def mixture_log_q(self, lq, mix):
        """log q_mix = log((1 - mix) q + mix 2^-n) from log q (tensor or array)."""
        lu = math.log(mix) - self.n * math.log(2.0)
        if isinstance(lq, torch.Tensor):
            return torch.logaddexp(lq + math.log1p(-mix), torch.full_like(lq, lu))
        return np.logaddexp(np.asarray(lq) + math.log1p(-mix), lu)

    def log_q(self, x_bf16):
        x_bf16 = self._input(x_bf16)
        batch = int(x_bf16.shape[0])
        buf = self._buffers(batch)
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().rgs_mlp_logq(batch, self.n, self.hidden, _p(x_bf16), *self._wargs(),
                                               _p(buf["logq"]), _p(buf["h1"]), _p(buf["h2"]), _p(buf["z"]),
                                               self._stream()))
        return buf["logq"]

    def state(self):
        """Host copies of the masters, masks and bf16 weights (for the CPU oracle)."""
        return {"w": [w.cpu().numpy() for w in self.w], "b": [b.cpu().numpy() for b in self.b],
                "masks": [m.cpu().numpy() for m in self.masks],
                "wb": [w.to(torch.float32).cpu().numpy() for w in self.wb]}


def calibrate_envelope(logp, logq, quantile=1.0, slack=1.0):
    """log c from held-out exact samples: the given quantile of log p - log q plus log(slack),
    and the estimated deficit D = E_p[max(0, 1 - c q / p)] on the same samples."""
    r = np.asarray(logp) - np.asarray(logq)
    log_c = float(np.quantile(r, quantile) + math.log(slack))
    deficit = float(np.mean(np.maximum(0.0, 1.0 - np.exp(log_c - r))))
    return log_c, deficit


def rejection_sample(p_fn, propose_fn, log_c, count, rng, max_rounds=1000, margin=1e-3, recheck_fn=None):
    """Accept x ~ q iff u < min(1, p(x) / (c q(x))), in batches, until ``count`` accepts.

    ``propose_fn(round) -> (bits uint8 [B, n] qubit order, log q [B])``; ``p_fn(bits) -> p``
    (complex64 scan); ``recheck_fn(bits) -> p`` (FP64 scan) for the decisions within
    ``margin`` (relative) of the threshold.  Returns accepted rows and statistics."""
    acc_bits, acc_p = [], []
    proposals = violations = rechecked = flips = 0
    start = time.perf_counter()
    for r in range(max_rounds):
        bits, logq = propose_fn(r)
        p = np.asarray(p_fn(bits), dtype=np.float64)
        if not np.all(np.isfinite(p)):
            raise ArithmeticError("Invalid target probability")
        ratio = np.exp(np.log(np.maximum(p, 1e-300)) - logq - log_c)
        acc = np.minimum(ratio, 1.0)
        u = rng.random(len(p))
        keep = u < acc
        violations += int(np.sum(ratio > 1.0))
        near = np.abs(u - acc) < margin * np.maximum(acc, 1e-300)
        if recheck_fn is not None and near.any():
            p64 = np.asarray(recheck_fn(bits[near]), dtype=np.float64)
            acc64 = np.minimum(np.exp(np.log(np.maximum(p64, 1e-300)) - logq[near] - log_c), 1.0)
            keep64 = u[near] < acc64
            flips += int(np.sum(keep64 != keep[near]))
            rechecked += int(near.sum())
            keep[near] = keep64
            p[near] = p64
        proposals += len(p)
        acc_bits.append(bits[keep])
        acc_p.append(p[keep])
        if sum(len(a) for a in acc_bits) >= count:
            break
    bits = np.concatenate(acc_bits)[:count]
    p = np.concatenate(acc_p)[:count]
    n = bits.shape[1]
    elapsed = time.perf_counter() - start
    return bits, p, {"proposals": proposals, "accepted": len(bits), "acceptance": len(bits) / max(1, proposals),
                     "envelope_violations": violations, "fp64_rechecked": rechecked, "fp64_flips": flips,
                     "linear_xeb": float((2.0 ** n) * p.mean() - 1) if len(p) else None, "seconds": elapsed}


def capped_rejection(scan_oracle, rng, count, cap=1.0, max_proposals=100000, recheck=None, batch=1024):
    """The reference's capped-probability sampler (``W/rejection_sampler.py:10-29``): per
    proposal, n uniform bits then one uniform; accept iff u < min(2^n p / cap, 1).  Same RNG
    call order as the reference; p(x) is evaluated in batches.  Output is distributed as
    min(2^n p, cap), not Born.  Returns (records, summary)."""
    n = scan_oracle.n
    records, accepted = [], 0
    total = 0
    while accepted < count and total < max_proposals:
        rows, us = [], []
        for _ in range(min(batch, max_proposals - total)):
            rows.append(rng.integers(0, 2, n))
            us.append(float(rng.random()))
        bits = np.array(rows, dtype=np.uint8)
        p = scan_oracle.probabilities(bits)
        scaled = (2.0 ** n) * p
        if not np.all(np.isfinite(scaled)):
            raise ArithmeticError("Invalid target probability")
        acc = np.minimum(scaled / cap, 1.0)
        u = np.array(us)
        if recheck is not None:
            near = np.abs(u - acc) < 1e-3 * np.maximum(acc, 1e-300)
            if near.any():
                p[near] = recheck.probabilities(bits[near])
                scaled = (2.0 ** n) * p
                acc = np.minimum(scaled / cap, 1.0)
        for i in range(len(bits)):
            keep = bool(u[i] < acc[i]) and accepted < count
            rec = {"proposal": total, "bitstring_q0_left": "".join(map(str, bits[i])), "probability_raw": float(p[i]),
                   "xeb_contribution": float(scaled[i] - 1), "acceptance_probability": float(acc[i]),
                   "acceptance_uniform": float(u[i]), "accepted": keep}
            if keep:
                rec["sample"] = accepted
                accepted += 1
            records.append(rec)
            total += 1
            if accepted >= count:
                break
    z = np.array([r["xeb_contribution"] for r in records if r["accepted"]])
    summary = {"completed": accepted == count, "accepted": accepted, "proposals": total,
               "acceptance_fraction": accepted / total if total else 0.0,
               "xeb": float(z.mean()) if len(z) else None}
    return records, summary
