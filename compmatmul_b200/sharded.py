"""k-sharded compressed product over several GPUs (one process per GPU).

The compressed product is linear in its rank-1 terms:

    p_t = IFFT( sum_k FFT(CS1_t(a_k)) * FFT(CS2_t(b_k)) )      (matmul_fft.hpp:70-112)

(and the same with the WHT, matmul_fwht.hpp:70-100), and the inverse
transform is linear too.  So when rank r holds rows [k_r, k_{r+1}) of AT and
B -- its slice of the inner index -- the sketch of its slice, computed with
the same (d, b, seed, hash), is the slice's share of p, and the sketch of the
whole product is the sum over ranks: one all-reduce of d x b doubles (4.7 MB
at d = 9, b = 2^16) after each rank's local sketch.  Recovery (decompression
or top-K) then runs on any rank from the reduced p.

On GPUs the reduction is NCCL over NVLink; the local sketches are this
package's kernels (device.compressed_product).  The split and the reduction
are plain torch.distributed calls, so they also run on gloo ranks on the CPU.
"""
from __future__ import annotations


def slice_bounds(n_inner, world, rank):
    """The contiguous inner-index range [k0, k1) of `rank` out of `world`:
    near-equal shares, the first n_inner % world ranks one row longer."""
    base, extra = divmod(int(n_inner), int(world))
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def reduce_sketch(p_local, group=None):
    """Sums the ranks' slice sketches in place (all-reduce, SUM): afterwards
    every rank holds the sketch of the whole product."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(p_local, op=dist.ReduceOp.SUM, group=group)
    return p_local


def compressed_product(AT_slice, B_slice, d, b, seed, variant="fft", hash=None, group=None):
    """Sketch p (d x b float64, on this rank's GPU) of the whole product from
    this rank's slice of the inner index (AT_slice: rows k0..k1 of AT, same
    for B), then summed over the ranks of `group`."""
    from . import device
    return reduce_sketch(device.compressed_product(AT_slice, B_slice, d, b, seed, variant, hash), group)
