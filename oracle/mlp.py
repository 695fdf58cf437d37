"""NumPy FP32 oracle of the edge-scoring MLP (no reference counterpart).

Restates the numerics of `tsp_gpu_clean_b200/csrc/mlp.cu` with the same BF16 rounding
points (round to nearest even): inputs and weights used in BF16, FP32 accumulation, the
first hidden layer stored in BF16, the output-layer gradient rounded to BF16 before the
W2^T product. Used by the GPU tests as the gradient check.

Test infrastructure only (see the package docstring).
"""

from __future__ import annotations

import numpy as np

H, KX, F = 64, 16, 5
O_W1 = 0
O_B1 = O_W1 + KX * H
O_W2 = O_B1 + H
O_B2 = O_W2 + H * H
O_W3 = O_B2 + H
O_B3 = O_W3 + H
COUNT = O_B3 + 1


def bf16(x: np.ndarray) -> np.ndarray:
  b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
  r = ((b >> 16) & 1) + 0x7FFF
  return ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
  W1 = p[O_W1:O_B1].reshape(KX, H)
  return W1, p[O_B1:O_W2], p[O_W2:O_B2].reshape(H, H), p[O_B2:O_W3], p[O_W3:O_B3], p[O_B3]


def forward(p: np.ndarray, x: np.ndarray):
  W1, b1, W2, b2, w3, b3 = unpack(p.astype(np.float32))
  xb = bf16(x.astype(np.float32))
  h1 = bf16(np.maximum(xb @ bf16(W1) + b1, 0))
  h2 = np.maximum(h1 @ bf16(W2) + b2, 0)
  logit = h2 @ bf16(w3) + b3
  return xb, h1, h2, logit.astype(np.float32)


def grads(p: np.ndarray, x: np.ndarray, y: np.ndarray, dh1_bf16: bool = False):
  """d(mean BCE with logits)/dp and the summed loss. `dh1_bf16`: dh1 enters dW1 and db1
  rounded to BF16, as in the tensor-core (tcgen05) training kernel of `csrc/mlp_tc.cu`."""
  W1, b1, W2, b2, w3, b3 = unpack(p.astype(np.float32))
  xb, h1, h2, logit = forward(p, x)
  E = x.shape[0]
  prob = 1.0 / (1.0 + np.exp(-logit.astype(np.float64)))
  d = ((prob - y) / E).astype(np.float32)
  dh2 = bf16(d[:, None] * bf16(w3)[None, :] * (h2 > 0))
  dh1 = (dh2 @ bf16(W2).T) * (h1 > 0)
  if dh1_bf16:
    dh1 = bf16(dh1.astype(np.float32))
  g = np.zeros(COUNT, dtype=np.float64)
  g[O_W1 : O_W1 + F * H] = (xb[:, :F].T.astype(np.float64) @ dh1).ravel()
  g[O_B1:O_W2] = dh1.sum(0)
  g[O_W2:O_B2] = (h1.T.astype(np.float64) @ dh2).ravel()
  g[O_B2:O_W3] = dh2.sum(0)
  g[O_W3:O_B3] = h2.T.astype(np.float64) @ d
  g[O_B3] = d.sum()
  lg = logit.astype(np.float64)
  loss = float(np.sum(np.maximum(lg, 0) - lg * y + np.log1p(np.exp(-np.abs(lg)))))
  return g, loss


def adam(p, g, m, v, step, lr=3e-3, b1=0.9, b2=0.999, eps=1e-8):
  g = g.astype(np.float32).copy()
  g[O_W1 + F * H : O_B1] = 0.0
  m = b1 * m + (1 - b1) * g
  v = b2 * v + (1 - b2) * g * g
  c1, c2 = 1 - b1**step, 1 - b2**step
  upd = lr * (m / c1) / (np.sqrt(v / c2) + eps)
  upd[O_W1 + F * H : O_B1] = 0.0
  return (p - upd).astype(np.float32), m, v
