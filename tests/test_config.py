"""config.json handling of the C++ host mirror (BatchDenoiser::factory,
batch_denoiser.cpp:36-118), read through the C ABI.  No GPU needed."""

import json

import pytest


def write(tmp_path, obj):
    p = tmp_path / "config.json"
    p.write_text(json.dumps(obj))
    return p


BASE = {
    "inputFolder": "/data/in",
    "outputFolder": "/data/out",
    "globalParams": {
        "patchWidthDim": 12, "patchHeightDim": 12, "slidingWidth": 4, "slidingHeight": 4, "atoms": 256,
        "ompIter": 5, "ksvdIter": 1, "B&W": True, "speckle": False, "type": "CUDA_K_GESVDJ",
        "minOmpIterBatch": 0, "subImageWidthDim": 0, "subImageHeightDim": 0,
    },
    "files": [
        {"name": "a.pgm", "ref": "a_ref.pgm"},
        {"name": "b.pgm", "patchWidthDim": 8, "patchHeightDim": 8, "atoms": 64, "speckle": True,
         "type": "CUDA_K_SM100A", "ksvdIter": 3, "noiseVariance": 12.5, "precision": "FP16"},
        {"name": "c.pgm", "type": "no-such-engine", "subImageWidthDim": 512, "subImageHeightDim": 280},
    ],
}


def test_globals_and_overrides(ksvd, built_lib, tmp_path):
    e = ksvd.batch_config(write(tmp_path, BASE))
    assert len(e) == 3
    a, b, c = e
    assert (a["patch_width_dim"], a["patch_height_dim"], a["sliding_width"], a["sliding_height"]) == (12, 12, 4, 4)
    assert (a["atoms"], a["omp_iter"], a["ksvd_iter"]) == (256, 5, 1)
    assert a["type"] == ksvd.CUDA_K_GESVDJ and a["speckle"] == 0 and a["bw"] == 1
    # per-file overrides
    assert (b["patch_width_dim"], b["atoms"], b["ksvd_iter"], b["speckle"]) == (8, 64, 3, 1)
    assert b["type"] == ksvd.CUDA_K_SM100A
    assert b["noise_variance"] == 12.5 and b["precision"] == ksvd.PREC_FP16_RESCORE
    # unknown type -> 0 (std::map::operator[] default), sub-image overrides
    assert c["type"] == ksvd.CUDA_K_GESVD
    assert (c["sub_image_width_dim"], c["sub_image_height_dim"]) == (512, 280)


def test_paths(ksvd, built_lib, tmp_path):
    a, b, c = ksvd.batch_config(write(tmp_path, BASE))
    # <out>/<pw>_<ph>_<name> (batch_denoiser.cpp:96), ref = <in>/<ref>
    assert a["input"] == "/data/in/a.pgm"
    assert a["output"] == "/data/out/12_12_a.pgm"
    assert b["output"] == "/data/out/8_8_b.pgm"
    assert a["ref"] == "/data/in/a_ref.pgm"
    assert b["ref"] == "/data/in/"  # no ref: PSNR is reported as -1


def test_missing_globals_use_reference_defaults(ksvd, built_lib, tmp_path):
    e = ksvd.batch_config(write(tmp_path, {"inputFolder": "i", "outputFolder": "o",
                                           "files": [{"name": "x.pgm"}]}))
    (x,) = e
    # denoisingLib.h:44-56
    assert (x["patch_width_dim"], x["sliding_width"], x["atoms"], x["ksvd_iter"], x["omp_iter"]) == (8, 2, 256, 10, 5)


def test_bad_config(ksvd, built_lib, tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{ not json")
    assert built_lib.ksvd_batch_count(str(p).encode()) == -1
    assert built_lib.ksvd_batch_count(str(tmp_path / "missing.json").encode()) == -1
    with pytest.raises(ksvd.KsvdError):
        ksvd.batch_config(p)


def test_comments_and_escapes(ksvd, built_lib, tmp_path):
    p = tmp_path / "c.json"
    p.write_text('{ // comment\n "inputFolder": "in\\u0041", "outputFolder": "o", "files": [{"name": "q\\"x.pgm"}]}')
    (x,) = ksvd.batch_config(p)
    assert x["input"] == 'inA/q"x.pgm'
