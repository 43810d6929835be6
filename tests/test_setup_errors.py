"""STIR's set-up errors of the ray-tracing matrix, raised by b200rt_create on the host before any device work.

Each case breaks one rule that ProjMatrixByBinUsingRayTracing / DataSymmetriesForBins_PET_CartesianGrid enforce
and checks the status and STIR's message.  No GPU is needed: the checks run before the device is touched.
"""
import ctypes
import dataclasses

import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G


def _create(geo):
    lib = _abi.load_library()
    out = ctypes.c_void_p()
    st = lib.b200rt_create(ctypes.byref(geo), 0, ctypes.byref(out))
    msg = lib.b200rt_last_error(None).decode()
    if out.value:
        lib.b200rt_destroy(out)
    return st, msg


def _small(**image_changes):
    pdi, img = G.small_3d_pet()
    img = dataclasses.replace(img, **image_changes)
    return G.make_geometry(pdi, img)


@pytest.mark.parametrize("origin", [(0.0, 1.0, 0.0), (0.0, 0.0, -0.5)])
def test_shifted_xy_origin(origin):
    # ProjMatrixByBinUsingRayTracing.cxx:276-277
    st, msg = _create(_small(origin=origin))
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert msg == "ProjMatrixByBinUsingRayTracing sadly doesn't support shifted x/y origin yet"


def test_z_origin_not_a_multiple_of_the_plane_spacing():
    # DataSymmetriesForBins_PET_CartesianGrid.cxx: the z shift needs the origin on a plane
    st, msg = _create(_small(origin=(1.0, 0.0, 0.0)))  # half of the 2 mm plane spacing
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert "the z origin should be a multiple of the plane separation" in msg


def test_z_spacing_not_the_ring_spacing_over_an_integer():
    # DataSymmetriesForBins_PET_CartesianGrid.cxx:70-79
    st, msg = _create(_small(voxel_size=(1.5, 4.0, 4.0)))  # 4 mm rings / 1.5 mm planes
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert "z-grid spacing equal to the ring spacing of the scanner divided by an integer" in msg


def test_axial_sampling_not_an_integer_multiple_of_the_plane_spacing():
    """Span 3 samples half the 4 mm ring spacing axially; planes of 4/3 mm divide the ring spacing but not the
    2 mm sampling.  ProjMatrixByBinUsingRayTracing's per-bin check (num_lors_per_axial_pos an integer,
    ProjMatrixByBinUsingRayTracing.cxx:669-681) guards the same rule, but set-up builds the symmetries first
    (:280-286) and their check (DataSymmetriesForBins_PET_CartesianGrid.cxx:92-105) fires before any bin is
    computed, in STIR as here."""
    pdi, img = G.small_3d_pet()
    pdi = G.ProjDataInfoCTI(pdi.scanner, 3, 7, 144, 64)
    img = dataclasses.replace(img, nz=22, voxel_size=(4.0 / 3.0, 4.0, 4.0))
    st, msg = _create(G.make_geometry(pdi, img))
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert msg == ("DataSymmetriesForBins_PET_CartesianGrid can currently only support z-grid spacing equal to the "
                   "sinogram spacing divided by an integer")


def test_unsupported_symmetry_setting():
    pdi, img = G.small_3d_pet()
    geo = G.make_geometry(pdi, img, symmetries=(True, True, True, True, False))
    st, msg = _create(geo)
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert "do_symmetry_shift_z=0" in msg


def test_valid_geometry_passes_the_host_checks():
    """A valid geometry gets past every host check; without a GPU it then stops at the device."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: creation would succeed")
    pdi, img = G.small_3d_pet()
    st, msg = _create(G.make_geometry(pdi, img))
    assert st != _abi.OK
    assert "origin" not in msg and "sampling" not in msg and "symmetr" not in msg, msg
