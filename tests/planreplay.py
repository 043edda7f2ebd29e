"""Numpy replay of a host-only plan (test helper).

Walks the chunk list exactly as the streaming kernel does (per CTA, per
chunk: partial = D[:, cols] @ g * scale, accumulated over the chunks of an
item and written at its last chunk) so the layout, the chunking and the LPT
schedule can be checked on a machine without a GPU.
"""
import numpy as np

K_FIRST, K_LAST = 1, 2


def decode(w):
    w = np.asarray(w, dtype=np.int64) & 0xFFFFFFFF
    data_off = int(w[0] | (w[1] << 32))
    scale = float(np.array([w[6]], dtype=np.uint32).view(np.float32)[0])
    flags = int(w[7])
    nseg = (flags >> 8) & 0xF
    cols = [int(w[12] & 0xFFFF), int(w[12] >> 16), int(w[13] & 0xFFFF), int(w[13] >> 16)]
    segs = [(int(np.int32(np.uint32(w[8 + k]))), cols[k], (flags >> (16 + k)) & 1) for k in range(nseg)]
    return dict(data_off=data_off, ncols=int(w[2]), hpad=int(w[3]), rows=int(w[4]), out_off=int(w[5]),
                scale=scale, flags=flags, segs=segs)


def run_phase(plan, xsrc, tsrc, out, dtype=np.float64):
    chunks, cta, data = plan["chunks"], plan["cta_ptr"], plan["data"]
    for b in range(len(cta) - 1):
        acc = None
        for i in range(cta[b], cta[b + 1]):
            d = decode(chunks[i])
            if d["flags"] & K_FIRST:
                acc = np.zeros(d["hpad"], dtype=dtype)
            if d["ncols"]:
                D = data[d["data_off"]:d["data_off"] + d["ncols"] * d["hpad"]].reshape(d["ncols"], d["hpad"]).T
                g = np.concatenate([(tsrc if src else xsrc)[off:off + n] for off, n, src in d["segs"]])
                assert g.size == d["ncols"]
                acc += (D.astype(dtype) @ g.astype(dtype)) * dtype(d["scale"])
            if d["flags"] & K_LAST:
                out[d["out_off"]:d["out_off"] + d["rows"]] = acc[:d["rows"]]
    return out


def replay(h, x_perm, precision="fp64", transposed=False):
    """y (permuted ordering) = H x_perm, replaying h's plan (h finalized with plan_only)."""
    p1 = h.plan_export(precision, 1, transposed)
    p2 = h.plan_export(precision, 2, transposed)
    info = h.info()
    t = np.zeros(max(1, info["sum_rank"]))
    run_phase(p1, x_perm, t, t)
    n_out = h.n_cols if transposed else h.n_rows
    y = np.full(n_out, np.nan)
    run_phase(p2, x_perm, t, y)
    return y
