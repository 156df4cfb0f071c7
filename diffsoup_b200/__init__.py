"""diffsoup_b200: B200-native differentiable triangle-soup rasterize-and-shade.

Drop-in for the rasterize/shade API of kenji-tojo/diffsoup
(python/diffsoup/__init__.py:11-25): the same public names with the same
signatures and tensor layouts, backed by hand-written sm_100a kernels in
libdiffsoup_b200.so.  `step` adds the batched, graph-captured training step,
`optimize` the fused VectorAdam / Adam updates that follow it, `viewer` the
headless inference render of the viewer's deferred shading, `remesh` the
soup subdivision of the resampling step.
"""

from __future__ import annotations

from . import _core
from . import optimize
from . import remesh
from . import viewer
from . import visibility
from ._core import __version__
from .rasterize import (
    count_triangle_ids,
    edge_grad,
    encode_view_dir,
    encode_view_dir_sh2,
    opacity_aux_loss,
)
from .point3d import (
    nn_spacing,
    remove_unreferenced_vertices_from_soup,
    triangle_soup_from_points,
)
from .remesh import (
    expand_by_index,
    split_triangle_soup,
    split_triangle_soup_clip,
    split_triangle_soup_clip_until,
    split_triangle_soup_until,
)
from .multires import (
    ColorMLP,
    accumulate_to_level,
    build_multires_triangle_color,
    feats_at_level,
    multires_triangle_color,
    rasterize_multires_triangle_alpha,
)

__all__ = [
    "ColorMLP",
    "accumulate_to_level",
    "build_multires_triangle_color",
    "count_triangle_ids",
    "edge_grad",
    "encode_view_dir",
    "encode_view_dir_sh2",
    "expand_by_index",
    "feats_at_level",
    "multires_triangle_color",
    "nn_spacing",
    "opacity_aux_loss",
    "rasterize_multires_triangle_alpha",
    "remove_unreferenced_vertices_from_soup",
    "split_triangle_soup",
    "split_triangle_soup_clip",
    "split_triangle_soup_clip_until",
    "split_triangle_soup_until",
    "triangle_soup_from_points",
]
