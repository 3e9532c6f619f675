"""CPU restatement of the row-shard merge protocol (test infrastructure).

The device steps of ``mlxlearn_b200.sharding.RowShardOps`` restated on CPU
tensors so that the exchange protocol (all-gather of the per-shard lists,
flagging of cross-shard near ties, all-reduce of exact keys, exact resolve)
can run on gloo ranks and be checked against the oracle:

* search: the oracle's exact kNN over the shard's rows;
* merge: the k-way merge of csrc/shards.cu, same flag rule;
* keys: S(q, x) * 2^298 as a Python integer (every float32 is a multiple of
  2^-149), split into ten 64-bit limbs;
* resolve: the first k by (exact key, global row).
"""
from __future__ import annotations

import numpy as np
import torch

import oracle

KEY_LIMBS = 10


class CpuShard:
    """A shard's rows, standing in for a device index."""

    def __init__(self, X):
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        self.n_samples = self.X.shape[0]


def shard_eps(d: int) -> float:
    u = 2.0 ** -53
    g = (d + 2) * u / (1.0 - (d + 2) * u)
    return 2 * g + 4 * u


def exact_key(q, x) -> int:
    s = 2.0 ** 149
    return sum((int(float(a) * s) - int(float(b) * s)) ** 2 for a, b in zip(q, x))


def to_limbs(v: int):
    out = []
    for _ in range(KEY_LIMBS):
        w = v & ((1 << 64) - 1)
        out.append(w - (1 << 64) if w >= 1 << 63 else w)
        v >>= 64
    return out


def from_limbs(ws) -> int:
    return sum((int(w) & ((1 << 64) - 1)) << (64 * i) for i, w in enumerate(ws))


class CpuRowShardOps:
    def search(self, shard, Q, k):
        d, i = oracle.knn(shard.X, Q.numpy(), k, nthreads=2)
        return torch.from_numpy(d), torch.from_numpy(i)

    def merge(self, D, I, k, d, self_offset):
        S, m, k_in = I.shape
        eps = shard_eps(d)
        Dn, In = D.numpy(), I.numpy()
        out_d = np.empty((m, k), np.float64)
        out_i = np.empty((m, k), np.int64)
        flags = np.zeros(m, np.int32)
        for q in range(m):
            self_row = self_offset + q if self_offset >= 0 else -2
            head = [0] * S
            for p in range(k):
                best = None
                for s in range(S):
                    while head[s] < k_in and In[s, q, head[s]] == self_row:
                        head[s] += 1
                    if head[s] >= k_in or In[s, q, head[s]] < 0:
                        continue
                    c = (Dn[s, q, head[s]], In[s, q, head[s]])
                    if best is None or c < best[1]:
                        best = (s, c)
                s0, (bd, bi) = best
                for s in range(S):
                    if s == s0 or head[s] >= k_in or In[s, q, head[s]] < 0:
                        continue
                    if bd * (1 + eps) >= Dn[s, q, head[s]] * (1 - eps):
                        flags[q] = 1
                out_d[q, p], out_i[q, p] = bd, bi
                head[s0] += 1
        return torch.from_numpy(out_d), torch.from_numpy(out_i), torch.from_numpy(flags)

    def keys(self, shard, row_offset, Q, I, flagged, keys):
        S, m, k_in = I.shape
        Qn, In = Q.numpy(), I.numpy()
        for f, q in enumerate(flagged.tolist()):
            for c in range(S * k_in):
                g = int(In[c // k_in, q, c % k_in])
                if row_offset <= g < row_offset + shard.n_samples:
                    keys[f, c] = torch.tensor(to_limbs(exact_key(Qn[q], shard.X[g - row_offset])))

    def resolve(self, D, I, k, self_offset, flagged, keys, out_d, out_i):
        S, m, k_in = I.shape
        for f, q in enumerate(flagged.tolist()):
            self_row = self_offset + q if self_offset >= 0 else -2
            cands = []
            for c in range(S * k_in):
                g = int(I[c // k_in, q, c % k_in])
                if g < 0 or g == self_row:
                    continue
                cands.append((from_limbs(keys[f, c].tolist()), g, float(D[c // k_in, q, c % k_in])))
            cands.sort(key=lambda t: (t[0], t[1]))
            for p, (_, g, dist) in enumerate(cands[:k]):
                out_i[q, p] = g
                out_d[q, p] = dist


def planted_rows(rng, n, d, n_shards):
    """Rows with cross-shard exact duplicates: the last shard's first rows copy
    rows of the first shard, so ties between shards must break by global row."""
    X = rng.standard_normal((n, d)).astype(np.float32)
    bounds = np.linspace(0, n, n_shards + 1).astype(int)
    last = bounds[-2]
    X[last:last + 20] = X[:20]
    return X, bounds


def oracle_radius_local(shard, Q, radius, need_distance, sort_results):
    """The oracle's radius search over a shard's rows, as a RadiusCSR."""
    from mlxlearn_b200.radius_result import RadiusCSR

    ip, ii, dd = oracle.radius(shard.X, Q, radius, sort_results=sort_results, nthreads=2)
    return RadiusCSR(ip, ii, dd if need_distance else None)
