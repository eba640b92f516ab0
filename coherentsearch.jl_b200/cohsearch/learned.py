"""The learned block proposal (no counterpart in the reference).

A small network scores each block of the band from its incoherent power-sum
features (``Engine.block_features``, cs_block_features).  The blocks whose
score reaches a threshold -- the proposed ones and the ones the network is
unsure of -- are re-searched by the coherent search (``Engine.
search_blocks_raw``, cs_search_blocks), which keeps the final word: every
reported candidate is the coherent search's, and recall is measured against
the full search's candidates.

The network (2*nharms -> 256 -> 256 -> 1, ReLU, BF16 weights, FP32
accumulation) runs and trains through the library's own kernels
(cs_mlp_forward, cs_mlp_backward, cs_adam_step); torch only holds the device
buffers.  Training labels come from the coherent search itself: a block is
positive when it holds a candidate above the threshold.
"""
import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _lib


class ProposalMLP:
    """Parameters (FP32 masters and their BF16 copies), Adam state and the
    training / inference calls of the proposal network."""

    def __init__(self, din: int, dh: int = 256, seed: int = 0, device: int = 0):
        import torch
        self.lib = _lib.load()
        self.din, self.dh, self.device = int(din), int(dh), int(device)
        self.dev = torch.device("cuda", self.device)
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        shapes = {"w1": (dh, din), "b1": (dh,), "w2": (dh, dh), "b2": (dh,), "w3": (dh,), "b3": (1,)}
        fan_in = {"w1": din, "w2": dh, "w3": dh}
        self.p = {}
        for k, s in shapes.items():
            if k.startswith("w"):
                t = torch.randn(s, generator=g) * np.sqrt(2.0 / fan_in[k])
                if k == "w3":
                    t *= 0.1
            else:
                t = torch.zeros(s)
            self.p[k] = t.to(self.dev, torch.float32).contiguous()
        self.bf = {k: torch.empty(self.p[k].shape, dtype=torch.int16, device=self.dev) for k in ("w1", "w2", "w3")}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.step = 0
        self._refresh_bf16()

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _refresh_bf16(self):
        for k in ("w1", "w2", "w3"):
            _lib.check(self.lib.cs_mlp_to_bf16(self.p[k].data_ptr(), self.bf[k].data_ptr(), self.p[k].numel(),
                                               self._stream()), None, "cs_mlp_to_bf16")

    def net(self):
        return _lib.cs_mlp(self.din, self.dh, self.bf["w1"].data_ptr(), self.p["b1"].data_ptr(),
                           self.bf["w2"].data_ptr(), self.p["b2"].data_ptr(), self.bf["w3"].data_ptr(),
                           self.p["b3"].data_ptr())

    def params_numpy(self):
        """FP32 masters on the host (for the oracle)."""
        return {k: v.detach().cpu().numpy().copy() for k, v in self.p.items()}

    def forward(self, x):
        """(h1, h2, logits) of rows x (float32 CUDA tensor [n, din])."""
        import torch
        x = x.contiguous()
        n = x.shape[0]
        h1 = torch.empty((n, self.dh), dtype=torch.float32, device=self.dev)
        h2 = torch.empty((n, self.dh), dtype=torch.float32, device=self.dev)
        z = torch.empty(n, dtype=torch.float32, device=self.dev)
        net = self.net()
        _lib.check(self.lib.cs_mlp_forward(ctypes.byref(net), x.data_ptr(), n, h1.data_ptr(), h2.data_ptr(),
                                           z.data_ptr(), self._stream()), None, "cs_mlp_forward")
        return h1, h2, z

    def loss_and_grads(self, x, y, pos_weight: float):
        """Loss (a float) and the gradients (into self.g) of one batch."""
        import torch
        x = x.contiguous()
        y = y.to(self.dev, torch.float32).contiguous()
        n = x.shape[0]
        h1, h2, z = self.forward(x)
        dz = torch.empty(n, dtype=torch.float32, device=self.dev)
        dh1 = torch.empty((n, self.dh), dtype=torch.float32, device=self.dev)
        dh2 = torch.empty((n, self.dh), dtype=torch.float32, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        net = self.net()
        gr = _lib.cs_mlp_grads(*(self.g[k].data_ptr() for k in ("w1", "b1", "w2", "b2", "w3", "b3")))
        _lib.check(self.lib.cs_mlp_backward(ctypes.byref(net), x.data_ptr(), h1.data_ptr(), h2.data_ptr(),
                                            z.data_ptr(), y.data_ptr(), n, float(pos_weight), dz.data_ptr(),
                                            dh1.data_ptr(), dh2.data_ptr(), ctypes.byref(gr), loss.data_ptr(),
                                            self._stream()), None, "cs_mlp_backward")
        return loss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        arr = (_lib.cs_adam_param * 6)()
        for i, k in enumerate(("w1", "b1", "w2", "b2", "w3", "b3")):
            arr[i] = _lib.cs_adam_param(self.p[k].data_ptr(), self.bf[k].data_ptr() if k in self.bf else None,
                                        self.m[k].data_ptr(), self.v[k].data_ptr(), self.g[k].data_ptr(),
                                        self.p[k].numel())
        _lib.check(self.lib.cs_adam_step(arr, 6, float(lr), float(b1), float(b2), float(eps), self.step,
                                         self._stream()), None, "cs_adam_step")

    def fit(self, X, Y, epochs=8, batch=4096, lr=1e-3, pos_weight=None, seed=0):
        """Mini-batch Adam over (X [n, din] CUDA tensor, Y [n] 0/1); returns the
        mean loss per epoch.  pos_weight defaults to the class ratio."""
        import torch
        Y = Y.to(self.dev, torch.float32)
        npos = float(Y.sum().item())
        if pos_weight is None:
            pos_weight = max(1.0, (len(Y) - npos) / max(npos, 1.0))
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(len(Y), generator=g).to(self.dev)
            tot = torch.zeros(1, dtype=torch.float32, device=self.dev)
            nb = 0
            for s in range(0, len(Y), batch):
                idx = perm[s:s + batch]
                tot += self.loss_and_grads(X[idx], Y[idx], pos_weight)
                self.adam(lr)
                nb += 1
            hist.append(float(tot.item()) / max(nb, 1))
        return hist

    def scores(self, X, batch=1 << 16):
        """Scores (sigmoid of the logits) of rows X (CUDA tensor), numpy."""
        z = [self.forward(X[s:s + batch])[2].cpu().numpy() for s in range(0, X.shape[0], batch)]
        z = np.concatenate(z).astype(np.float64) if z else np.zeros(0)
        return 1.0 / (1.0 + np.exp(-z))


def block_labels(raw, nblocks, blocksize=2048, threshold=8.0):
    """1 for the blocks holding a candidate above `threshold` (any level)."""
    y = np.zeros(nblocks, np.float32)
    sel = raw[raw["metric"] > threshold]
    y[np.unique(sel["trial"] // blocksize)] = 1.0
    return y


def choose_threshold(scores, y, recall=0.995):
    """The largest score threshold keeping `recall` of the positive blocks."""
    pos = np.sort(np.asarray(scores)[np.asarray(y) > 0.5])
    if len(pos) == 0:
        return 0.5
    k = int(np.floor((1.0 - recall) * len(pos)))
    return float(pos[k]) * (1.0 - 1e-6)


@dataclass
class LearnedResult:
    cands: np.ndarray          # candidates of the re-searched blocks
    blocks: np.ndarray         # re-searched block indices
    nblocks: int               # blocks of the band
    ms_features: float
    ms_scores: float
    ms_search: float


def learned_search(engine, mlp, tau, lofreq, hifreq, lobin=100, blocksize=2048, threshold=None):
    """Features, scores and the coherent re-search of the blocks scoring >= tau
    (host wall times around each stage, each ending in a device sync)."""
    import torch
    t0 = time.perf_counter()
    X = engine.block_features(lofreq, hifreq, lobin, blocksize)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    s = mlp.scores(X)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    blocks = np.nonzero(s >= tau)[0].astype(np.int64)
    cands = engine.search_blocks_raw(blocks, lofreq, hifreq, lobin, blocksize, threshold)
    t3 = time.perf_counter()
    return LearnedResult(cands, blocks, int(X.shape[0]), 1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (t3 - t2))


def recall_of(found, full, threshold=8.0):
    """Fraction of `full`'s candidates above threshold that `found` holds (by trial and k)."""
    want = {(int(c["trial"]), int(c["k"])) for c in full[full["metric"] > threshold]}
    if not want:
        return 1.0
    got = {(int(c["trial"]), int(c["k"])) for c in found}
    return len(want & got) / len(want)
