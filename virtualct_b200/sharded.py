"""One slice over the ranks of a torch.distributed process group (no
counterpart in the reference, which runs one slice on one host).

    forward   each rank projects its share of the sinogram rows
              (vct_forward_views_dev) and reports their (max, min);
    exchange  one all-reduce combines (max, -min) with MAX: the global max
              normalises, the global min sets the noise clamp;
    normalise each rank normalises and adds noise to its own rows
              (vct_normalize_noise_rows_dev; noise keyed by view and
              channel, so it does not depend on the split);
    gather    one all-gather assembles the normalised sinogram on every rank;
    FBP       each rank filters the sinogram (a few tens of microseconds) and
              backprojects one band of the image (vct_fbp_band_dev); one
              all-reduce sums the disjoint bands.

Every pixel and every sinogram element is computed by one rank exactly as on
one GPU, so the pieced results equal vct_mbfpa_dev's and vct_fbp_dev's bit
for bit.  Collectives move 8 bytes, the sinogram and the image (1.9 MB and
1 MB at 800 x 609 and 512^2).  For many slices, independent replicas (one
slice per rank, no collective) are the faster layout; this one cuts the
latency of a single slice.
"""
from __future__ import annotations


def split(n: int, parts: int, i: int) -> tuple[int, int]:
    """Part i of [0, n) in `parts` contiguous, balanced pieces."""
    return n * i // parts, n * (i + 1) // parts


class ShardedSlice:
    def __init__(self, ctx, dist=None, group=None):
        """ctx: a Context with maps and spectrum set; dist: torch.distributed
        (initialised; NCCL for CUDA tensors) or None for a single rank.  The
        context is bound to torch's current CUDA stream, on which the
        collectives are ordered."""
        self.ctx, self.dist, self.group = ctx, dist, group
        if dist is not None and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.dist, self.rank, self.world = None, 0, 1

    def _bind_stream(self, device) -> None:
        import torch

        if device.type == "cuda":
            # torch's default stream has handle 0, which vct_set_stream reads as
            # "the context's own stream": name it as cudaStreamLegacy (1) instead
            h = torch.cuda.current_stream(device).cuda_stream
            self.ctx.set_stream(h if h else 1)

    def mbfpa(self, sigma: float, seed: int, out):
        """The normalised (noisy) sinogram [views][width] into `out` on every
        rank."""
        import torch

        self._bind_stream(out.device)
        g = self.ctx.geometry
        V, W, used = g.views, g.width, g.views // 2 * 2
        r0, r1 = split(V, self.world, self.rank)
        maxmin = torch.empty(2, dtype=torch.float32, device=out.device)
        self.ctx.forward_views_dev(min(r0, used), min(r1, used), out, maxmin)
        if r1 > used:  # rows past views/2*2 are zero, as the reference leaves them
            out[max(r0, used):r1].zero_()
        if self.dist is not None:
            t = torch.stack([maxmin[0], -maxmin[1]])
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
            maxmin = torch.stack([t[0], -t[1]]).contiguous()
        self.ctx.normalize_noise_rows_dev(out, r0, r1, maxmin, sigma, seed)
        if self.dist is not None:
            chunk = -(-V // self.world)  # equal pieces for the all-gather
            mine = torch.zeros((chunk, W), dtype=out.dtype, device=out.device)
            mine[: r1 - r0] = out[r0:r1]
            parts = [torch.empty_like(mine) for _ in range(self.world)]
            self.dist.all_gather(parts, mine, group=self.group)
            for i in range(self.world):
                a, b = split(V, self.world, i)
                if i != self.rank:
                    out[a:b] = parts[i][: b - a]
        return out

    def fbp(self, sino, img, filter: int = 1, in_mode: bool = False):
        """The FBP image [N][N] of `sino` into `img` on every rank."""
        self._bind_stream(img.device)
        nb = self.ctx.fbp_band_count()
        b0, b1 = split(nb, self.world, self.rank)
        img.zero_()
        self.ctx.fbp_band_dev(sino, b0, b1, img, filter=filter, in_mode=in_mode)
        if self.dist is not None:
            self.dist.all_reduce(img, op=self.dist.ReduceOp.SUM, group=self.group)
        return img
