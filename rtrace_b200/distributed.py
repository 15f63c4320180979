"""One frame split into row bands across ranks (one process per GPU).

Pixels of the reference's render are independent (src/renderer.rs:445-584:
every pixel seeds its own StdRng; src/renderer.rs:752-897: quincunx corners
are seeded by their grid position), so rank r renders a contiguous band of
rows with `Renderer.render_rows`, which traces the outline stencil's extra
rows itself, and the bands are gathered to the root.  No data moves between
ranks while they render; the only collective is the final gather of RGB8
rows to the root (width * rows * 3 bytes per rank).

With the NCCL backend the bands are rendered straight into CUDA tensors and
gathered over NVLink; with gloo (CPU tests) they are host tensors.
"""
import numpy as np
import torch
import torch.distributed as dist


def row_bands(height, world_size, row_costs=None):
    """Contiguous row bands [(begin, end), ...], one per rank, covering
    [0, height) in order.  Without costs the bands differ by at most one
    row; with per-row cost estimates (for instance ray counts from a
    previous frame) the cuts split the total cost evenly.  A rank may get an
    empty band when height < world_size."""
    if height < 0 or world_size < 1:
        raise ValueError("height must be >= 0 and world_size >= 1")
    if row_costs is None:
        base, extra = divmod(height, world_size)
        bands, y = [], 0
        for r in range(world_size):
            n = base + (1 if r < extra else 0)
            bands.append((y, y + n))
            y += n
        return bands
    c = np.asarray(row_costs, dtype=np.float64)
    if c.shape != (height,) or (c < 0).any():
        raise ValueError("row_costs must hold one non-negative cost per row")
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world_size):
        target = total * r / world_size
        y = int(np.searchsorted(cum, target, side="left"))
        cuts.append(min(max(y, cuts[-1]), height))
    cuts.append(height)
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


def gather_bands(band, bands, width, group=None, root=0):
    """Gathers every rank's band (a (rows, width, 3) uint8 tensor, rows =
    that rank's band height) to `root`, which returns the (height, width, 3)
    image as a numpy array; other ranks return None.  Bands are padded to the
    tallest band so that one gather of equal-sized buffers moves them; only
    the root receives (world - 1 bands cross the links, not world^2 as an
    all-gather would move)."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if len(bands) != world:
        raise ValueError("one band per rank expected")
    rows = bands[rank][1] - bands[rank][0]
    if tuple(band.shape) != (rows, width, 3) or band.dtype != torch.uint8:
        raise ValueError(f"rank {rank}: band must be a uint8 tensor of shape {(rows, width, 3)}")
    tallest = max(e - b for b, e in bands)
    padded = torch.zeros((tallest, width, 3), dtype=torch.uint8, device=band.device)
    padded[:rows] = band
    root_global = root if group is None else dist.get_global_rank(group, root)
    if rank != root:
        dist.gather(padded, None, dst=root_global, group=group)
        return None
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.gather(padded, parts, dst=root_global, group=group)
    return torch.cat([parts[r][:e - b] for r, (b, e) in enumerate(bands)], 0).cpu().numpy()


def render_frame(renderer, scene, group=None, root=0, row_costs=None, band_renderer=None):
    """Renders one frame across the ranks of `group`; the root returns the
    (height, width, 3) uint8 image, identical to renderer.render(scene) on
    one GPU, and the other ranks return None.

    band_renderer(begin, end) -> (rows, width, 3) uint8 tensor replaces the
    GPU band render (host tests use it to exercise the partition and gather
    without a GPU)."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    bands = row_bands(renderer.height, world, row_costs)
    b, e = bands[rank]
    if band_renderer is not None:
        band = band_renderer(b, e)
    else:
        dev = torch.device("cuda", scene._ctx.device)
        band = torch.empty((e - b, renderer.width, 3), dtype=torch.uint8, device=dev)
        if e > b:
            renderer.render_rows(scene, b, e, device_ptr=band.data_ptr())
    return gather_bands(band, bands, renderer.width, group=group, root=root)


def reduce_timings(times, counts, device=None, group=None):
    """Whole-job timing of a multi-rank run: every rank passes its own device
    times and work counts; all ranks get back (max over ranks of each time,
    sum over ranks of each count).  A job is as slow as its slowest rank and
    does the work of all of them."""
    t = torch.tensor([float(v) for v in times], dtype=torch.float64, device=device)
    n = torch.tensor([float(v) for v in counts], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    return t.tolist(), n.tolist()
