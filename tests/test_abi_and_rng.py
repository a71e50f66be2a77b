"""CPU checks of the C-ABI library: it loads, exports every function the
public headers declare, reports the absence of a GPU as a status, and its
counter RNG matches the published Philox-4x32-10 answers and the oracle's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(az_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert "az_gpu_produce_image" in names and "az_scene_generate" in names
    lib = az.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing


# Random123 known-answer vectors for philox4x32_10
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    c = np.array(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    az.lib().az_rng_philox4x32_10(c.ctypes.data, key[0], key[1], out.ctypes.data)
    assert tuple(int(x) for x in out) == want
    out2 = np.zeros(4, np.uint32)
    ol.port().azo_philox(c.ctypes.data, key[0], key[1], out2.ctypes.data)
    assert tuple(int(x) for x in out2) == want


def test_draws_match_oracle_keying():
    rng = np.random.default_rng(1)
    L = ol.port()
    for _ in range(2000):
        seed = int(rng.integers(0, 2**63))
        args = [int(x) for x in rng.integers(0, 2**32, size=3)] + [int(rng.integers(0, 20)), int(rng.integers(0, 64))]
        a = az.lib().az_rng_u01(seed, *args)
        b = L.azo_u01(seed, *args)
        assert a == b and 0.0 <= a < 1.0


def test_no_gpu_is_reported_as_a_status():
    if az.device_info(0) is not None:
        pytest.skip("a GPU is present")
    sc = az.generate_scene(az.SCENE_CORNELL, width=4, height=4, spp=1)
    with pytest.raises(az.AzError) as e:
        az.produce_image(sc)
    assert e.value.code == 7


def test_generated_scene_shapes():
    sc = az.generate_scene(az.SCENE_DENSE_MESH, width=32, height=32, spp=4, detail=2)
    assert sc.triangle_count == 12 + 20 * 4 ** 2
    assert sc.resolution() == (32, 32) and sc.sample_count() == 4 and sc.max_depth() == 8
    c0 = az.generate_scene(az.SCENE_CORNELL)
    assert c0.resolution() == (256, 256) and c0.sample_count() == 16 and c0.max_depth() == 5
    assert c0.triangle_count == 12 and c0.sphere_count == 2
    # interior: three rooms, every surface tessellated at `detail` cells per metre
    # (panels of two triangles per cell), 36 clutter boxes and the 2-triangle light
    it = az.generate_scene(az.SCENE_INTERIOR, width=32, height=18, spp=4, detail=4)
    assert it.resolution() == (32, 18) and it.max_depth() == 10
    assert 20000 < it.triangle_count < 40000
    assert it.triangle_count % 2 == 0


def test_launch_variant_count_matches_header():
    import re
    hdr = open(os.path.join(REPO, "include", "azimuth_gpu.h")).read()
    assert int(re.search(r"#define AZ_LAUNCH_VARIANTS (\d+)", hdr).group(1)) == az.LAUNCH_VARIANTS
