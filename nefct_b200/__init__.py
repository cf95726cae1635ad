"""nefct_b200: B200-native (sm_100a) projector hot path of nefct (CT-NEF).

Cone-beam ray-driven (slab-split "Siddon") forward projector, its exact
transpose and the reference's own backprojection, the LOR projector pair,
FDK (cosine/Parker weighting, ramp filtering, voxel-driven weighted
backprojection), the distance-driven projector pair and the cpp/deform
trilinear warp -- hand-written CUDA
kernels behind the C ABI of include/nefct_b200.h, wrapped as torch ops with
autograd and as drop-ins for the reference's python operators.

Importing needs no GPU; running any operator does (there is no CPU path).
"""
from . import _lib
from ._lib import NefctError
from .base import nef_class
from .geometry import (DetectorConfig, DetectorDirectAConfig, DetectorDirectBConfig, ScannerConfig,
                       ScannerConfig3D)
from .data import (Image, Image3D, Image3DT, ProjectionSequence3D, all_one_image, all_zero_image,
                   ellipsoid_phantom, phantom, random_ellipsoids)
from . import ops
from .ops import ConeBeam, DDGeometry, backproject, dd_project, project, warp
from .functions import (FDK, SART, BackProject3D, BackProject3DT, ConjGrad, Project3D, Project3DT,
                        WarpDeformer, cone_beam)
from . import cc
from . import recon
from .io import json_dump, json_dumps, json_load, json_loads, load, save

__version__ = "0.1.0"
