"""Configuration codes of the fused-stage variants (bbw_autotune /
bbw_set_config): W | ops_in_smem << 8 | pipelined << 9 | (E == 16) << 10."""
import pytest

from bbwadg_b200.solver import decode_config, encode_config


def test_codes_round_trip():
    for tile in (32, 16):
        for warps in (8, 16):
            for ops in (False, True):
                for pipe in (False, True):
                    code = encode_config(warps, ops, pipe, tile)
                    d = decode_config(code)
                    assert (d["warps"], d["ops_in_smem"], d["pipelined"], d["tile"]) == \
                        (warps, ops, pipe, tile)
                    assert d["code"] == code


def test_code_layout():
    assert encode_config(8, True, False) == 8 | 1 << 8
    assert encode_config(16, False, True, 16) == 16 | 1 << 9 | 1 << 10


def test_bad_tile_is_rejected():
    with pytest.raises(ValueError):
        encode_config(8, True, True, 64)
