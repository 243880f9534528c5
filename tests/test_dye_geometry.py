"""The fused dye kernel's tiles whose traces stay under one texel skip the window bounds
tests (s2d_dye.cuh, dye_cta_passes<TX, true>); the library's host-side self-check walks
every tile of every grid and dye size and confirms that such traces read only velocity
cells and dye texels inside the tile's windows.  Host code only: no GPU."""
import pytest

SIZES = [32, 64, 128, 256, 512, 1024, 2048, 4096]


@pytest.mark.parametrize("scale", [1, 2, 4])
@pytest.mark.parametrize("n", SIZES)
def test_fast_dye_tiles_stay_inside_their_windows(pkg, n, scale):
    lib = pkg.lib()
    rc = lib.s2d_dye_fast_path_check(n, scale)
    assert rc == 0, lib.s2d_last_error().decode()


@pytest.mark.parametrize("n,scale", [(48, 2), (8192, 2), (256, 3)])
def test_fast_path_check_rejects_unsupported_sizes(pkg, n, scale):
    assert pkg.lib().s2d_dye_fast_path_check(n, scale) < 0
