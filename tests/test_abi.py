"""The C ABI library loads and exports every entry point include/*.h declares;
argument errors are reported before any GPU work (runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

import klitho as K

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(kl_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) >= 25
    for must in ("kl_socs_forward", "kl_tcc_build", "kl_topk_eig", "kl_hopkins_image",
                 "kl_create_source", "kl_create_mask", "kl_write_kernel_info"):
        assert must in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_symbol(name):
    lib = ctypes.CDLL(K.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_version_and_error_string():
    assert K.lib().kl_version() >= 10000
    assert isinstance(K.lib().kl_last_error(), bytes)


def test_unsupported_geometry_rejected_before_gpu():
    # any period is accepted; a SOCS grid 4N+1 above 256, or above half the
    # period, is refused on the host before any device work
    with pytest.raises(K.KLError) as e:
        K.SocsPlan(8192, 8192, 70, 70, 2)
    assert e.value.code == K.KL_ERR_UNSUPPORTED
    with pytest.raises(K.KLError) as e:
        K.SocsPlan(256, 256, 40, 40, 2)
    assert e.value.code == K.KL_ERR_UNSUPPORTED
    with pytest.raises(K.KLError) as e:
        K.SocsPlan(1024, 1024, 13, 13, 0)
    assert e.value.code == K.KL_ERR_INVALID


def test_tcc_plan_argument_errors_before_gpu():
    import numpy as np
    src = K.createSource(41, "Annular", 0.6, 0.9)
    with pytest.raises(K.KLError) as e:
        K.TccPlan(src, 1.35, 0.0, 512, 512, n_medium=1.0)  # NA > n: phase undefined
    assert e.value.code == K.KL_ERR_INVALID
    with pytest.raises(K.KLError) as e:
        K.TccPlan(np.zeros((41, 41), np.float32), 0.8, 0.0, 512, 512)  # empty source
    assert e.value.code == K.KL_ERR_INVALID
