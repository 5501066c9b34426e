"""B-spline node-field interpolation on the device (include/psum_interp.h).

The free functions of PSuM's src/field/higher_order_interp.hpp:196-247 with
the order as an argument: ``interp_B_spline`` (value), ``interp_diff_B_spline``
(gradient) and ``add_back_B_spline`` (deposit), applied to n positions at
once.  Positions are a (dim, n) float64 CUDA tensor (SoA), fields a float64
CUDA tensor of prod(cells + 1) nodes, last dimension fastest.  Work runs on
torch's current stream, so it is ordered with the surrounding torch work.
"""
import ctypes as C

from ._lib import GridDesc, check, lib


def grid_desc(grid):
    """psum_pic_grid_desc of a ``simple_grid`` (or of a ``GridDesc``, returned as is)."""
    if isinstance(grid, GridDesc):
        return grid
    g = GridDesc()
    g.dim = grid.dim
    for a in range(3):
        g.cells[a] = grid.cells[a] if a < grid.dim else 1
        g.lower[a] = grid.lower[a] if a < grid.dim else 0.0
        g.upper[a] = grid.upper[a] if a < grid.dim else 1.0
        g.periodic[a] = 0
    return g


def _check_args(order, pos, field, dim):
    import torch
    if order not in (1, 2, 3, 4):
        raise ValueError("order must be 1, 2, 3 or 4")
    for t in (pos, field):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise TypeError("positions and fields must be contiguous float64 CUDA tensors")
    if pos.dim() != 2 or pos.shape[0] != dim:
        raise ValueError(f"positions must have shape ({dim}, n)")


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _skip_ptr(skipped):
    """Device address of the optional 64-bit skip counter."""
    if skipped is None:
        return None
    import torch
    if not (isinstance(skipped, torch.Tensor) and skipped.is_cuda and skipped.dtype in (torch.int64, torch.uint64)
            and skipped.numel() >= 1):
        raise TypeError("skipped must be a 64-bit integer CUDA tensor with at least one element")
    return skipped.data_ptr()


def interp_B_spline(order, grid, pos, field, skipped=None):
    """Interpolated field values at the positions (interp_B_spline<order>); a
    position without support gives NaN and increments ``skipped`` (a uint64 /
    int64 CUDA tensor of one element) when given."""
    import torch
    g = grid_desc(grid)
    _check_args(order, pos, field, g.dim)
    n = pos.shape[1]
    out = torch.empty(n, dtype=torch.float64, device=pos.device)
    check(lib().psum_interp_bspline(C.byref(g), order, n, pos.data_ptr(), field.data_ptr(), out.data_ptr(),
                                    _skip_ptr(skipped), _stream()))
    return out


def interp_diff_B_spline(order, grid, pos, field, skipped=None):
    """Gradient of the interpolant at the positions, (dim, n)
    (interp_diff_B_spline<order>; E = -gradient for a potential)."""
    import torch
    g = grid_desc(grid)
    _check_args(order, pos, field, g.dim)
    n = pos.shape[1]
    out = torch.empty((g.dim, n), dtype=torch.float64, device=pos.device)
    check(lib().psum_interp_diff_bspline(C.byref(g), order, n, pos.data_ptr(), field.data_ptr(), out.data_ptr(),
                                         _skip_ptr(skipped), _stream()))
    return out


def add_back_B_spline(order, grid, pos, weight, field, scratch=None, skipped=None):
    """field += weight * W(pos) summed over the positions (add_back_B_spline<order>),
    in place; ``scratch`` optionally supplies prod(cells + 1) 64-bit words."""
    g = grid_desc(grid)
    _check_args(order, pos, field, g.dim)
    n = pos.shape[1]
    check(lib().psum_add_back_bspline(C.byref(g), order, n, pos.data_ptr(), float(weight), field.data_ptr(),
                                      None if scratch is None else scratch.data_ptr(), _skip_ptr(skipped),
                                      _stream()))


def deposit_bits(n):
    """Fraction bits of the deposit's fixed point for n positions."""
    b = C.c_int()
    check(lib().psum_bspline_deposit_bits(n, C.byref(b)))
    return b.value
