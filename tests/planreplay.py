"""Numpy replay of a host-only plan (test helper).

Walks the chunk list exactly as the streaming kernel does (per CTA, per
chunk: partial = D[:, cols] @ (g * segment scale), accumulated over the chunks
of an item and written at its last chunk, phase-1 outputs times the per-t
scale) so the layout, the chunking and the LPT schedule can be checked on a
machine without a GPU.
"""
import numpy as np

K_FIRST, K_LAST = 1, 2
WORDS = 28


def decode(w):
    w = np.asarray(w, dtype=np.int64) & 0xFFFFFFFF
    data_off = int(w[0] | (w[1] << 32))
    flags = int(w[6])
    nseg = (flags >> 8) & 0xF
    cols = []
    for k in range(8):
        word = int(w[16 + k // 2])
        cols.append((word >> (16 * (k % 2))) & 0xFFFF)
    scales = np.array(w[20:28], dtype=np.uint32).view(np.float32)
    segs = [(int(np.int32(np.uint32(w[8 + k]))), cols[k], (flags >> (16 + k)) & 1, float(scales[k]))
            for k in range(nseg)]
    return dict(data_off=data_off, ncols=int(w[2]), hpad=int(w[3]), rows=int(w[4]), out_off=int(w[5]),
                flags=flags, segs=segs)


def chunk_matrix(data, d, tiled):
    """hpad x ncols block of a chunk from the flat data array."""
    hp, nc = d["hpad"], d["ncols"]
    if not tiled:
        return data[d["data_off"]:d["data_off"] + nc * hp].reshape(nc, hp).T
    ng = (nc + 7) // 8
    t = data[d["data_off"]:d["data_off"] + ng * 8 * hp].reshape(ng, hp // 8, 8, 8)  # [cgroup, rgroup, c%8, r%8]
    M = t.transpose(1, 3, 0, 2).reshape(hp, ng * 8)
    return M[:, :nc]


def run_phase(plan, xsrc, tsrc, out, tiled=False, t_scale=None):
    chunks, cta, data = plan["chunks"], plan["cta_ptr"], plan["data"]
    for b in range(len(cta) - 1):
        acc = None
        for i in range(cta[b], cta[b + 1]):
            d = decode(chunks[i])
            if d["flags"] & K_FIRST:
                acc = np.zeros(d["hpad"])
            if d["ncols"]:
                D = chunk_matrix(data, d, tiled)
                g = np.concatenate([(tsrc if src else xsrc)[off:off + n] * sc for off, n, src, sc in d["segs"]])
                assert g.size == d["ncols"]
                acc += D @ g
            if d["flags"] & K_LAST:
                r = acc[:d["rows"]]
                if t_scale is not None:
                    r = r * t_scale[d["out_off"]:d["out_off"] + d["rows"]]
                out[d["out_off"]:d["out_off"] + d["rows"]] = r
    return out


def replay(h, x_perm, precision="fp64", transposed=False):
    """y (permuted ordering) = H x_perm, replaying h's plan (h finalized with plan_only)."""
    import ctypes as C

    from bigwham_dev_b200 import _capi as A

    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    tiled = precision == "bf16"
    ts = None
    if tiled:
        n = C.c_int64()
        A.check(A.lib().bw_plan_tscale(h._h, int(transposed), C.byref(n), None), h._h)
        buf = (C.c_float * n.value)()
        A.check(A.lib().bw_plan_tscale(h._h, int(transposed), C.byref(n), buf), h._h)
        ts = np.frombuffer(buf, dtype=np.float32).astype(np.float64)
    info = h.info()
    t = np.zeros(max(1, info["sum_rank"]))
    run_phase(p1, x_perm, t, t, tiled, ts)
    n_out = h.n_cols if transposed else h.n_rows
    y = np.full(n_out, np.nan)
    run_phase(p2, x_perm, t, y, tiled)
    return y
