"""Row sharding of the 2D-torus exchange across ranks (one process per GPU).

The torus of N sub-filters has dx = 2^floor(log2 sqrt N) columns and
dy = N / dx rows; sub-filter b sits at column b % dx, row b // dx.  Each
sub-filter's weakest 4t slots take the top-t particles of its right, left,
bottom and top neighbours (slot m-1-j-k*t from neighbour k, the torus routing
of the single-GPU engine).  With `world` ranks each rank owns dy / world
consecutive rows.  Left/right neighbours are always on the same rank; the top
neighbour of a rank's first row is the last row of the rank above, and the
bottom neighbour of its last row is the first row of the rank below.  Per
step every rank therefore sends two halos -- the top-t particles of its first
row (to the rank above) and of its last row (to the rank below), dx * t
particles each -- and receives two: one point-to-point exchange with each
neighbouring rank, no collective over the particles.  The global estimate
needs one small all-reduce of the FP64 partials.

`halo_exchange` works with any torch.distributed backend (gloo on CPU tensors,
NCCL on CUDA tensors).
"""
import numpy as np


def torus_dims(N):
    dx = 1
    while (2 * dx) * (2 * dx) <= N:
        dx *= 2
    return dx, N // dx


class TorusShard:
    """Rank `rank`'s block of rows of an N-sub-filter torus (m particles each, t transferred)."""

    def __init__(self, N, m, t, world, rank):
        self.N, self.m, self.t, self.world, self.rank = N, m, t, world, rank
        self.dx, self.dy = torus_dims(N)
        if self.dx * self.dy != N:
            raise ValueError("torus exchange needs N = dx * dy (N=%d)" % N)
        if self.dy % world:
            raise ValueError("%d torus rows do not split over %d ranks" % (self.dy, world))
        if 5 * t > m:
            raise ValueError("torus exchange needs 5 t <= m")
        self.rows = self.dy // world
        self.row0 = rank * self.rows
        self.up = (rank - 1) % world    # owns the row above row0
        self.down = (rank + 1) % world  # owns the row below the last row

    @property
    def first_subfilter(self):
        return self.row0 * self.dx

    @property
    def num_subfilters(self):
        return self.rows * self.dx

    def halos_out(self, sorted_state, sorted_keys):
        """(to_up, to_down): top-t particles of the first and last local row,
        each (state [S, dx*t], keys [dx*t]) from the local sorted copy
        (state [S, n*m], keys [n*m], sub-filters in local order)."""
        m, t, dx = self.m, self.t, self.dx
        out = []
        for r in (0, self.rows - 1):
            idx = np.array([(r * dx + c) * m + j for c in range(dx) for j in range(t)], np.int64)
            out.append((sorted_state[:, idx], sorted_keys[idx]))
        return out[0], out[1]

    def sources(self):
        """For every local sub-filter b and slot x < 4t (slot m-1-x): (where, index),
        where 0 = local sorted copy (particle index), 1 = halo from the rank
        above, 2 = halo from the rank below (index into the halo)."""
        m, t, dx, dy = self.m, self.t, self.dx, self.dy
        src = np.zeros((self.num_subfilters, 4 * t, 2), np.int64)
        for lb in range(self.num_subfilters):
            gb = self.first_subfilter + lb
            x, y = gb % dx, gb // dx
            for k in range(4):
                if k == 0:
                    fy, fx = y, (x + 1) % dx
                elif k == 1:
                    fy, fx = y, (x - 1) % dx
                elif k == 2:
                    fy, fx = (y + 1) % dy, x
                else:
                    fy, fx = (y - 1) % dy, x
                for j in range(t):
                    local_row = fy - self.row0
                    if 0 <= local_row < self.rows:
                        src[lb, k * t + j] = (0, (local_row * dx + fx) * m + j)
                    elif k == 2:
                        src[lb, k * t + j] = (2, fx * t + j)
                    else:
                        src[lb, k * t + j] = (1, fx * t + j)
        return src

    def apply_exchange(self, sorted_state, sorted_keys, halo_up, halo_down):
        """The exchange on the local sorted copy: returns (state, keys) with each
        sub-filter's weakest 4t slots replaced (the pre-resampling particles)."""
        m, t = self.m, self.t
        st, ks = sorted_state.copy(), sorted_keys.copy()
        src = self.sources()
        halos = {1: halo_up, 2: halo_down}
        for lb in range(self.num_subfilters):
            for x in range(4 * t):
                where, i = src[lb, x]
                dst = lb * m + m - 1 - x
                if where == 0:
                    st[:, dst] = sorted_state[:, i]
                    ks[dst] = sorted_keys[i]
                else:
                    st[:, dst] = halos[where][0][:, i]
                    ks[dst] = halos[where][1][i]
        return st, ks


def halo_exchange(dist, shard, to_up, to_down):
    """Send this rank's first-row halo up and last-row halo down, receive the
    neighbours' (tuples of torch tensors, e.g. (state, keys), the same shapes
    on every rank); returns (from_up, from_down).
    Sends are posted down-halo first and receives up-halo first, so that with
    two ranks (the same peer above and below) the messages pair up in order
    on backends without tags; the tags say the same for those that use them.
    With one rank both halos are the rank's own rows."""
    import torch
    if shard.world == 1:
        return to_down, to_up
    from_up = tuple(torch.empty_like(x) for x in to_up)
    from_down = tuple(torch.empty_like(x) for x in to_down)
    ops = []
    for x in to_down:
        ops.append(dist.P2POp(dist.isend, x.contiguous(), shard.down, tag=1))
    for x in to_up:
        ops.append(dist.P2POp(dist.isend, x.contiguous(), shard.up, tag=2))
    for x in from_up:
        ops.append(dist.P2POp(dist.irecv, x, shard.up, tag=1))
    for x in from_down:
        ops.append(dist.P2POp(dist.irecv, x, shard.down, tag=2))
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    return from_up, from_down


class ShardedFilter:
    """This rank's rows of a torus-exchange filter of config.num_subfilters
    sub-filters, stepped together with the other ranks' rows (pf_shard_*, one
    process per GPU).  Per step: sampling on every rank; two halo blocks of
    halo_bytes to each neighbouring rank (halo_exchange: the first row's top t
    to the rank above, the last row's to the rank below); resampling; one
    all_gather of the group rows (ceil(n / 32) rows of 32 doubles and the
    groups' winner states per rank) from which every rank forms the same
    estimate.  The ranks' particles and the estimate equal the whole filter's
    on one GPU bit for bit.  The rows split evenly: dy / world rows per rank,
    each rank's first sub-filter a multiple of 32.  Halos and group rows travel
    as CPU tensors on gloo and as CUDA tensors on NCCL."""

    def __init__(self, dist, model, params, config=None, **cfg):
        from . import FilterShard, default_config
        self.dist = dist
        self.world, self.rank = dist.get_world_size(), dist.get_rank()
        c = config if config is not None else default_config(**cfg)
        self.geom = TorusShard(c.num_subfilters, c.particles_per_subfilter, c.num_transfer, self.world, self.rank)
        g = self.geom
        self.shard = FilterShard(model, params, g.row0, g.row0 + g.rows, config=c)
        import torch
        self.device = (torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl"
                       else torch.device("cpu"))

    def set_initial_state(self, state):
        self.shard.set_initial_state(state)

    def particles(self):
        """This rank's particles, num_state x (its sub-filters x m)."""
        return self.shard.particles()

    def _t(self, a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def step(self, inp):
        """One step of the whole filter; returns its estimate (ESTIMATE_DTYPE record)."""
        sh, dist = self.shard, self.dist
        sh.sample(inp)
        to_up, to_down = sh.halo_out(1), sh.halo_out(0)
        from_up, from_down = halo_exchange(dist, self.geom, (self._t(to_up),), (self._t(to_down),))
        sh.halo_in(0, from_up[0].cpu().numpy())    # the row above this rank's first row
        sh.halo_in(1, from_down[0].cpu().numpy())  # the row below its last row
        sh.resample()
        rows, states = sh.group_rows()
        r, st = self._t(rows), self._t(states)
        all_r = [r.new_empty(r.shape) for _ in range(self.world)]
        all_s = [st.new_empty(st.shape) for _ in range(self.world)]
        dist.all_gather(all_r, r)
        dist.all_gather(all_s, st)
        return sh.estimate(np.concatenate([x.cpu().numpy() for x in all_r]),
                           np.concatenate([x.cpu().numpy() for x in all_s]))

    def close(self):
        self.shard.close()


# ---------------------------------------------------------------------------
# Moving served filters between ranks (elasticity).  A filter is snapshotted
# on its rank (pf_server_snapshot: int64 header {magic, model, particles,
# sub-filters}, then particles, MTGP32 stream words and the update count),
# sent, opened on the destination with the same model, parameters and count,
# and restored there (pf_server_restore); its next updates give the results
# it would have given at home.
# ---------------------------------------------------------------------------
SNAPSHOT_MAGIC = 0x5046535256534E31


def snapshot_header(buf):
    """(model, particles, sub-filters) from a pf_server_snapshot buffer; raises
    ValueError when the buffer is not one."""
    h = np.frombuffer(bytes(buf[:32]), dtype=np.int64)
    if len(h) != 4 or int(h[0]) != SNAPSHOT_MAGIC:
        raise ValueError("not a served-filter snapshot")
    return int(h[1]), int(h[2]), int(h[3])


def plan_moves(loads):
    """Rebalance served filters over ranks by particle count.  loads[r] is rank
    r's list of (filter id, particles).  Greedy: while moving some filter from
    the most loaded rank to the least loaded one lowers the larger of the two
    loads, move the largest such filter.  Returns [(src, dst, filter id)]."""
    per = [dict(l) for l in loads]
    moves = []
    while len(per) > 1:
        tot = [sum(p.values()) for p in per]
        hi = max(range(len(per)), key=lambda r: (tot[r], -r))
        lo = min(range(len(per)), key=lambda r: (tot[r], r))
        best = None
        for fid, n in sorted(per[hi].items(), key=lambda kv: (-kv[1], kv[0])):
            if max(tot[hi] - n, tot[lo] + n) < tot[hi]:
                best = (fid, n)
                break
        if best is None:
            break
        fid, n = best
        del per[hi][fid]
        per[lo][fid] = n
        moves.append((hi, lo, fid))
    return moves


def send_filter(dist, snap, dst):
    """Send one snapshot (bytes) to rank dst: its length, then its bytes."""
    import torch
    payload = torch.from_numpy(np.frombuffer(bytes(snap), dtype=np.uint8).copy())
    dist.send(torch.tensor([payload.numel()], dtype=torch.int64), dst, tag=3)
    dist.send(payload, dst, tag=4)


def recv_filter(dist, src):
    """Receive one snapshot sent by send_filter from rank src (bytes)."""
    import torch
    n = torch.zeros(1, dtype=torch.int64)
    dist.recv(n, src, tag=3)
    payload = torch.empty(int(n.item()), dtype=torch.uint8)
    dist.recv(payload, src, tag=4)
    return payload.numpy().tobytes()
