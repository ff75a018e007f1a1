"""The reference's MatrixFilter restated in numpy — TEST INFRASTRUCTURE ONLY.

core/task/cpu_task/cpu_subiso.cu:237-277 with the scalar helpers of
core/task/gpu_task/kernel/kernel_matrix_ops.cu:
  * SimdSquaredDifferenceSIMD (:76-87): diff = a - b; c = diff * diff
  * CPUOnlyMatMult with transposed B (:431-447): C[j] = sum_p A[p] * B[j*k + p],
    p ascending, one float32 rounding per product and per sum
  * CPUOnlyMatAdd (:486-505), ReluSIMD (:122-132): x > 0 ? x : 0
  * SigmoidSIMD (:157-181): 1.0f / (1.0f + expf(-x))
  * reject when the sigmoid is below 0.1 (cpu_subiso.cu:271).
numpy float32 array arithmetic rounds every operation to float32 and never
fuses a multiply with an add, which is the arithmetic of those scalar loops;
the only freedom left is the last bit of exp, so ``keep`` also reports the
candidates whose sigmoid lies within 1e-6 of the threshold.
"""
from __future__ import annotations

import numpy as np


def logits(query_emb, data_emb, w1, b1, w2, b2, u: int, vs) -> np.ndarray:
    """z2 = W2 . relu(W1 . (e_u - e_v)^2 + b1) + b2 for every v in vs (float32)."""
    f = np.float32
    eu = np.asarray(query_emb, dtype=f)[u]
    ev = np.asarray(data_emb, dtype=f)[np.asarray(vs, dtype=np.int64)]
    w1 = np.asarray(w1, dtype=f)
    hidden, dim = w1.shape
    d = eu[None, :] - ev
    sim = d * d
    z = np.zeros((len(ev), hidden), dtype=f)
    for p in range(dim):
        z = z + sim[:, p:p + 1] * w1[None, :, p]
    z = z + np.asarray(b1, dtype=f).reshape(1, hidden)
    z = np.where(z > 0, z, f(0))
    w2 = np.asarray(w2, dtype=f).reshape(hidden)
    z2 = np.zeros(len(ev), dtype=f)
    for j in range(hidden):
        z2 = z2 + z[:, j] * w2[j]
    return z2 + np.asarray(b2, dtype=f).reshape(-1)[0]


def keep(query_emb, data_emb, w1, b1, w2, b2, u: int, vs):
    """(keep, uncertain): keep[i] when the filter keeps (u, vs[i]); uncertain[i]
    when its sigmoid is within 1e-6 of 0.1 (the decision then depends on the
    last bit of exp)."""
    z2 = logits(query_emb, data_emb, w1, b1, w2, b2, u, vs)
    s = np.float32(1.0) / (np.float32(1.0) + np.exp(-z2))
    s64 = 1.0 / (1.0 + np.exp(-z2.astype(np.float64)))
    return ~(s < np.float32(0.1)), np.abs(s64 - 0.1) < 1e-6
