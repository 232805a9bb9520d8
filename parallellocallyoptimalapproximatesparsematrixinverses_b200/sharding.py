"""Column sharding of the SPAI iteration over several GPUs: the exchanges
that keep a sharded run bit-identical to a single-GPU run.

Every op of the iteration except the global scalars (and the transpose of
the drop step) is column-local, so the columns of M, R, Z and P can be split
into contiguous ranges, one per rank, with A replicated.  A global scalar on
one GPU is the fixed tree over the per-column partial sums: chunks of 4096
values, each folded by 256 lanes (lane t adds values t, t + 256, ... in
order) and a butterfly over the lanes, repeated over the chunk sums until
one value is left (ops.cu, TreeChunkKernel).  Cutting the columns only at
multiples of 4096 makes each rank's first-level chunk sums exactly the
global ones, so

    rank r: chunk sums of its columns           (on its device)
    all ranks: all_gather of the chunk sums     (n / 4096 values per scalar)
    every rank: the upper levels of the tree    (the same arithmetic)

gives every rank the single-GPU value, bit for bit, with one small
all-gather per set of scalars.  `shard_columns` makes such a cut and
`sharded_tree_sums` does the exchange and the upper levels (torch.distributed;
NCCL on GPUs, gloo on the host).  `tree_chunk_sums` / `tree_sum` restate the
device tree on the host for the upper levels.

The global budget's drop selects the `drop` smallest (score, offset) keys
over all candidates by a 16-pass radix select (ops.cu, RadixHistKernel /
RadixDecideKernel).  Sharded, each rank histograms its own candidates and
one all-reduce of the 256 bins per pass gives every rank the same digit:
`sharded_drop_cutoff` restates that select with the exchange, offsets being
the candidates' global column-major positions (rank order = column order).

The drop step's symmetrisation 0.5 (M + M^T) needs, in every rank's columns,
the rows of M that other ranks hold: `sharded_transpose` sends each entry to
the rank that owns its row with one all-to-all and returns this rank's
columns of M^T (rows ascending), device-agnostic torch code (NCCL moves
device tensors directly, over NVLink; no multicast).
"""
from __future__ import annotations

import numpy as np

TREE_LANES = 256
TREE_CHUNK = 4096


def shard_columns(n: int, world: int, align: int = TREE_CHUNK):
    """Contiguous column ranges [start, stop) for `world` ranks, cut only at
    multiples of `align` (the last range takes the remainder); ranks beyond
    the number of chunks get empty ranges."""
    if n < 0 or world <= 0 or align <= 0:
        raise ValueError("n >= 0, world > 0 and align > 0 are required")
    chunks = -(-n // align)
    bounds = [min(n, (chunks * r // world) * align) for r in range(world + 1)]
    bounds[-1] = n
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def _butterfly(lanes: np.ndarray) -> float:
    """The lane butterfly of one chunk: strides 128 .. 1, s[t] = s[t] + s[t ^ stride]."""
    s = lanes.copy()
    t = np.arange(TREE_LANES)
    stride = TREE_LANES // 2
    while stride >= 1:
        s = s + s[t ^ stride]
        stride //= 2
    return float(s[0])


def tree_chunk_sums(values) -> np.ndarray:
    """First level of the fixed tree: one sum per chunk of 4096 values."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    count = v.size
    chunks = -(-count // TREE_CHUNK)
    out = np.empty(chunks, dtype=np.float64)
    for c in range(chunks):
        part = np.zeros(TREE_CHUNK, dtype=np.float64)
        block = v[c * TREE_CHUNK:(c + 1) * TREE_CHUNK]
        part[:block.size] = block
        lanes = np.zeros(TREE_LANES, dtype=np.float64)
        # lane t adds values t, t + 256, ... in order, starting from +0.0
        for m in range(TREE_CHUNK // TREE_LANES):
            lanes = lanes + part[m * TREE_LANES:(m + 1) * TREE_LANES]
        out[c] = _butterfly(lanes)
    return out


def tree_sum(values) -> float:
    """The whole fixed tree (+0.0 for no values)."""
    level = np.ascontiguousarray(values, dtype=np.float64)
    if level.size == 0:
        return 0.0
    while True:
        level = tree_chunk_sums(level)
        if level.size == 1:
            return float(level[0])


def sharded_tree_sums(local_chunk_sums, group=None, device=None):
    """Global tree sums from every rank's first-level chunk sums.

    local_chunk_sums: array of shape (scalars, chunks of this rank), the
    chunk sums of this rank's column range (cut by `shard_columns`).  The
    exchange runs on `device` (a CUDA device under NCCL; the host under
    gloo).  Returns the `scalars` global sums, identical on every rank and
    bit-identical to the single-device tree over all columns."""
    import torch
    import torch.distributed as dist
    device = torch.device("cpu") if device is None else torch.device(device)
    local = np.ascontiguousarray(np.atleast_2d(local_chunk_sums), dtype=np.float64)
    world = dist.get_world_size(group)
    # ranks may hold different chunk counts: exchange the counts, then pad to the longest
    count = torch.tensor([local.shape[1]], dtype=torch.int64, device=device)
    counts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    counts = [int(c.item()) for c in counts]
    longest = max(counts)
    padded = np.zeros((local.shape[0], longest), dtype=np.float64)
    padded[:, :local.shape[1]] = local
    pieces = [torch.zeros((local.shape[0], longest), dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(pieces, torch.from_numpy(padded).to(device), group=group)
    chunk_sums = np.concatenate([p.cpu().numpy()[:, :c] for p, c in zip(pieces, counts)], axis=1)
    out = []
    for row in chunk_sums:
        out.append(float(row[0]) if row.size == 1 else (0.0 if row.size == 0 else tree_sum(row)))
    return out


def sharded_transpose(col_offsets, row_indices, values, ranges, rank, group=None):
    """This rank's columns [start, stop) of M^T from this rank's columns of M.

    col_offsets / row_indices / values: the rank's columns of M as CSC (torch
    tensors; offsets local, from 0, rows global); ranges: every rank's
    (start, stop), as shard_columns gives.  Returns (col_offsets,
    row_indices, values) of the rank's columns of M^T, rows ascending in
    every column, on the inputs' device."""
    import torch
    import torch.distributed as dist
    start, stop = ranges[rank]
    device = values.device
    lengths = col_offsets[1:] - col_offsets[:-1]
    cols = torch.repeat_interleave(torch.arange(start, stop, dtype=torch.int64, device=device), lengths)
    rows = row_indices.to(torch.int64)
    # the owner of each entry's row, and the entries grouped by owner (stable, so column order holds)
    starts = torch.tensor([a for a, _ in ranges[1:]], dtype=torch.int64, device=device)
    owner = torch.bucketize(rows, starts, right=True)
    order = torch.argsort(owner, stable=True)
    rows, cols, vals = rows[order], cols[order], values[order]
    world = len(ranges)
    send_counts = torch.bincount(owner, minlength=world).to(torch.int64)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    send_splits = send_counts.tolist()
    recv_splits = recv_counts.tolist()
    total = int(sum(recv_splits))
    got_rows = torch.empty(total, dtype=torch.int64, device=device)
    got_cols = torch.empty(total, dtype=torch.int64, device=device)
    got_vals = torch.empty(total, dtype=values.dtype, device=device)
    dist.all_to_all_single(got_rows, rows.contiguous(), recv_splits, send_splits, group=group)
    dist.all_to_all_single(got_cols, cols.contiguous(), recv_splits, send_splits, group=group)
    dist.all_to_all_single(got_vals, vals.contiguous(), recv_splits, send_splits, group=group)
    # entry (i, j) of M is entry (j, i) of M^T: column i - start, row j
    n = int(ranges[-1][1])
    local_col = got_rows - start
    key = local_col * max(n, 1) + got_cols
    order = torch.argsort(key)
    out_rows = got_cols[order]
    out_vals = got_vals[order]
    counts = torch.bincount(local_col, minlength=stop - start)
    out_ptr = torch.zeros(stop - start + 1, dtype=torch.int64, device=device)
    out_ptr[1:] = torch.cumsum(counts, 0)
    return out_ptr, out_rows, out_vals


def ordered_bits(scores) -> np.ndarray:
    """The order-preserving unsigned image of FP64 scores (ops.cu OrderedBits):
    -0.0 and +0.0 map alike, and unsigned order equals numeric order."""
    v = np.ascontiguousarray(scores, dtype=np.float64).copy()
    v[v == 0.0] = 0.0
    u = v.view(np.uint64)
    negative = (u >> np.uint64(63)) == np.uint64(1)
    return np.where(negative, ~u, u | np.uint64(1 << 63))


def sharded_drop_cutoff(keys, offset_base: int, drop: int, group=None, device=None):
    """The cutoff (score bits, offset) of the `drop` smallest keys over all
    ranks: keys are this rank's ordered score bits (ordered_bits), its
    candidates holding global offsets offset_base, offset_base + 1, ...  Every
    rank returns the same pair; a candidate is dropped iff its (bits, offset)
    <= the cutoff, as on one GPU.  Raises ValueError on every rank unless
    0 < drop <= the number of candidates over all ranks (the device select's
    own check), so that no rank enters the radix passes alone."""
    import torch
    import torch.distributed as dist
    device = torch.device("cpu") if device is None else torch.device(device)
    hi = np.ascontiguousarray(keys, dtype=np.uint64)
    count = torch.tensor([hi.size], dtype=torch.int64, device=device)
    dist.all_reduce(count, group=group)
    total = int(count.item())
    if not 0 < int(drop) <= total:
        raise ValueError(f"drop count {int(drop)} must lie in [1, {total}] (the candidates over all ranks)")
    lo = np.arange(offset_base, offset_base + hi.size, dtype=np.uint64)
    prefix_hi = np.uint64(0)
    prefix_lo = np.uint64(0)
    remaining = int(drop)
    for step in range(16):
        shift = np.uint64(56 - 8 * (step % 8))
        if step < 8:
            mask = np.uint64(0) if step == 0 else np.uint64((0xFFFFFFFFFFFFFFFF << (int(shift) + 8)) & 0xFFFFFFFFFFFFFFFF)
            match = (hi & mask) == (prefix_hi & mask)
            digits = ((hi[match] >> shift) & np.uint64(0xFF)).astype(np.int64)
        else:
            mask = np.uint64(0) if step == 8 else np.uint64((0xFFFFFFFFFFFFFFFF << (int(shift) + 8)) & 0xFFFFFFFFFFFFFFFF)
            match = (hi == prefix_hi) & ((lo & mask) == (prefix_lo & mask))
            digits = ((lo[match] >> shift) & np.uint64(0xFF)).astype(np.int64)
        local = torch.from_numpy(np.bincount(digits, minlength=256).astype(np.int64)).to(device)
        dist.all_reduce(local, group=group)
        hist = local.cpu().numpy()
        cumulative = np.cumsum(hist)
        digit = int(np.searchsorted(cumulative, remaining))  # first bin whose running count reaches the rank
        below = int(cumulative[digit - 1]) if digit > 0 else 0
        if step < 8:
            prefix_hi |= np.uint64(digit) << shift
        else:
            prefix_lo |= np.uint64(digit) << shift
        remaining -= below
    return int(prefix_hi), int(prefix_lo)
