"""Numpy replay of a host-only plan (test helper).

Walks the chunk list exactly as the streaming kernel does (per CTA, per
chunk: partial = D[:, cols] @ g[g_off : g_off + ncols], accumulated over the
chunks of an item and written at its last chunk, phase-1 outputs times the
per-t scale), with the phase-2 gather array G2 rebuilt from its runs, so the
layout, the chunking and the LPT schedule can be checked on a machine without
a GPU.
"""
import ctypes as C

import numpy as np

K_FIRST, K_LAST = 1, 2
WORDS = 8


def decode(w):
    w = np.asarray(w, dtype=np.int64) & 0xFFFFFFFF
    return dict(data_off=int(w[0] | (w[1] << 32)), ncols=int(w[2]), hpad=int(w[3]), rows=int(w[4]),
                out_off=int(w[5]), flags=int(w[6]), g_off=int(np.int32(np.uint32(w[7]))))


def chunk_matrix(data, d, tiled):
    """hpad x ncols block of a chunk from the flat data array."""
    hp, nc = d["hpad"], d["ncols"]
    if not tiled:
        return data[d["data_off"]:d["data_off"] + nc * hp].reshape(nc, hp).T
    ng = (nc + 7) // 8
    t = data[d["data_off"]:d["data_off"] + ng * 8 * hp].reshape(ng, hp // 8, 8, 8)  # [cgroup, rgroup, c%8, r%8]
    return t.transpose(1, 3, 0, 2).reshape(hp, ng * 8)[:, :nc]


def run_phase(plan, gsrc, out, tiled=False):
    chunks, items, data = plan["chunks"], plan["item_ptr"], plan["data"]
    for b in range(len(items) - 1):
        acc = None
        for i in range(items[b], items[b + 1]):
            d = decode(chunks[i])
            if d["flags"] & K_FIRST:
                acc = np.zeros(d["hpad"])
            if d["ncols"]:
                acc += chunk_matrix(data, d, tiled) @ gsrc[d["g_off"]:d["g_off"] + d["ncols"]]
            if d["flags"] & K_LAST:
                out[d["out_off"]:d["out_off"] + d["rows"]] = acc[:d["rows"]]
    return out


def gather_runs(h, precision, transposed):
    from bigwham_dev_b200 import _capi as A

    n = C.c_int64()
    f = A.PRECISIONS[precision]
    A.check(A.lib().bw_plan_gather(h._h, f, int(transposed), C.byref(n), None), h._h)
    runs = np.zeros((n.value, 4), np.int32)
    A.check(A.lib().bw_plan_gather(h._h, f, int(transposed), C.byref(n), runs.ctypes.data), h._h)
    return runs


def build_g2(runs, x, t):
    cols = (runs[:, 2].view(np.uint32) & 0x7FFFFFFF).astype(np.int64)
    src = runs[:, 2].view(np.uint32) >> 31
    scale = runs[:, 3].view(np.float32).astype(np.float64)
    g2 = np.zeros(int((runs[:, 0] + cols).max()) if len(runs) else 0)
    for (dst, off), c, s, sc in zip(runs[:, :2].astype(np.int64), cols, src, scale):
        g2[dst:dst + c] = sc * (t if s else x)[off:off + c]
    return g2


def replay(h, x_perm, precision="fp64", transposed=False):
    """y (permuted ordering) = H x_perm, replaying h's plan (h finalized with plan_only)."""
    from bigwham_dev_b200 import _capi as A

    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    tiled = precision == "bf16"
    t = np.zeros(max(1, h.info()["sum_rank"]))
    run_phase(p1, x_perm, t, tiled)  # BF16: t unscaled; the G2 runs carry the block scales
    g2 = build_g2(gather_runs(h, precision, transposed), x_perm, t)
    y = np.full(h.n_cols if transposed else h.n_rows, np.nan)
    run_phase(p2, g2, y, tiled)
    return y


# --------------------------------------------------------------------------- matmat plan
def mm_tile(data, off, hpad, kc):
    """(hpad x kc) float64 matrix of a chunk stored in 8x8 BF16 tiles:
    element (i, c) at off + (c/8)*8*hpad + (i/8)*64 + (c%8)*8 + i%8."""
    words = data[off:off + kc * hpad].astype(np.uint32) << 16
    t = words.view(np.float32).astype(np.float64)
    # axes of the flat array: column group, row group, column in group, row in group
    t = t.reshape(kc // 8, hpad // 8, 8, 8)
    return t.transpose(1, 3, 0, 2).reshape(hpad, kc)


def _bf16(a):
    u = np.ascontiguousarray(a, dtype=np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def mm_replay(h, X_perm, transposed=False, check=None, round_operands=False):
    """Walks the matmat plan of a BW_PLAN_ONLY handle as the tensor-core kernel
    does, in float64: returns Y (permuted ordering, n_out x k).  With the
    operands kept exact the structure, not the rounding, is under test;
    round_operands=True rounds X and the phase-1 products T8 to BF16 as the
    kernel does.  check(chunk_words) is called on every chunk."""
    k = X_perm.shape[1]
    if k > 64:  # passes of 64 right-hand sides, as the kernel runs them
        return np.concatenate([mm_replay(h, X_perm[:, c:c + 64], transposed, check, round_operands)
                               for c in range(0, k, 64)], axis=1)
    n_in, n_out = (h.n_rows, h.n_cols) if transposed else (h.n_cols, h.n_rows)
    p1, p2 = h.mm_plan_export(1, transposed), h.mm_plan_export(2, transposed)
    ops = [np.zeros(((n_in + 7) // 8 * 8 + 32, 64)), np.zeros((p1["t8_len"] + 32, 64))]
    ops[0][:n_in, :k] = _bf16(X_perm) if round_operands else X_perm
    Y = np.zeros((n_out, k))
    for phase, pl in ((1, p1), (2, p2)):
        acc = None
        for w in pl["chunks"]:
            if check is not None:
                check(w)
            off = int(np.uint32(w[0])) | (int(np.uint32(w[1])) << 32)
            kc, hpad, rows, out_off, flags = int(w[2]), int(w[3]), int(w[4]), int(w[5]), int(np.uint32(w[6]))
            nr = (flags >> 8) & 0xFF
            B = []
            for r in range(nr):
                src, nrow = int(np.uint32(w[8 + 2 * r])), int(w[9 + 2 * r])
                B.append(ops[src >> 31][(src & 0x7FFFFFFF):(src & 0x7FFFFFFF) + nrow])
            B = np.concatenate(B, axis=0)
            if flags & 1:
                acc = np.zeros((hpad, 64))
            acc += mm_tile(pl["data"], off, hpad, kc) @ B
            if flags & 2:
                if phase == 1:
                    ops[1][out_off:out_off + rows] = _bf16(acc[:rows]) if round_operands else acc[:rows]
                else:
                    Y[out_off:out_off + rows] = acc[:rows, :k]
    return Y
