"""Multi-GPU helpers: one process per GPU, torch.distributed for the plumbing.

The path shards without a data-path exchange: a frame's samples split into
disjoint Z-Sobol index ranges (every rank draws its slice of the same
sequence: first_sample = its offset, sampler_spp = the frame's spp), so the
sum of the ranks' film sums is the single-GPU frame's film.  One all-reduce
of the film sums (NCCL over NVLink on GPUs, gloo on CPU) finishes the frame;
the adjoint's texel and emission gradients are summed the same way.
"""


def sample_range(spp, rank, world):
    """(first_sample, count) of rank's slice of spp samples (the first
    spp % world ranks take one extra)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("sample_range: bad rank or world size")
    base, extra = divmod(int(spp), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def split_params(params, rank, world):
    """A copy of a gzg_render_params (ctypes) record for rank's slice; None
    when the rank has no samples."""
    first, count = sample_range(params.spp, rank, world)
    if count == 0:
        return None
    p = type(params).from_buffer_copy(params)
    p.first_sample = params.first_sample + first
    p.sampler_spp = params.sampler_spp if params.sampler_spp > 0 else params.spp
    p.spp = count
    return p


def allreduce_films(tensors, group=None):
    """Sums film tensors (torch) over the ranks in place."""
    import torch.distributed as dist

    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


def render_frame(render_slice, params, films, group=None):
    """One frame over all ranks: render_slice(params_slice, films) adds this
    rank's samples to `films` (zeroed by the caller), then the film sums are
    all-reduced.  Every rank takes the same collective steps, also when its
    slice is empty."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    p = split_params(params, rank, world)
    if p is not None:
        render_slice(p, films)
    return allreduce_films(films, group)


def render_frame_device(renderer_factory, params, films, stream=None, group=None):
    """render_frame for a GPU scene: renderer_factory(params_slice) returns a
    Renderer (accel.Renderer) whose render(rgb, w, sq) adds the slice to the
    device films (rgb, w[, sq])."""
    def slice_fn(p, f):
        with renderer_factory(p) as r:
            r.render(f[0], f[1], f[2] if len(f) > 2 else None, stream=stream)

    return render_frame(slice_fn, params, films, group)


def allreduce_gradients(d_texels, d_emission, group=None):
    """Sums the adjoint's gradients over the ranks (each rank replayed its
    own sample slice)."""
    return allreduce_films([d_texels, d_emission], group)


__all__ = ["sample_range", "split_params", "allreduce_films", "render_frame", "render_frame_device",
           "allreduce_gradients"]
