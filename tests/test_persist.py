"""Model files in the reference's layouts (persist/schema.rs, json.rs,
envelope.rs, binary.rs): .bstr.json envelopes and .bstr binaries
(32-byte header, MessagePack named-map payload, 16-byte trailer with
CRC32C). CPU tests: the files are built here by hand or with an independent
MessagePack encoder, read through the C ABI and checked through the tree
accessors; the GPU round trip (trained models, predictions) is in
test_gpu_persist.py."""
import json
import pickle
import struct

import msgpack
import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n


def crc32c(b):
    return n.lib.bst_crc32c(bytes(b), len(b))


def test_crc32c_known_answers():
    # iSCSI (RFC 3720 B.4) vectors and the common check value
    assert crc32c(b"\x00" * 32) == 0x8A9136AA
    assert crc32c(b"\xff" * 32) == 0x62A8AB43
    assert crc32c(bytes(range(32))) == 0x46DD794E
    assert crc32c(bytes(range(31, -1, -1))) == 0x113FDB5C
    assert crc32c(b"123456789") == 0xE3069283


def stump(transform="identity"):
    """node 0: x0 < 0.5 (missing left) -> 1 else 2; leaves 1.0, 2.0."""
    return {"meta": {"num_features": 2, "num_groups": 1},
            "forest": {"trees": [{"num_nodes": 3, "split_indices": [0, 0, 0], "thresholds": [0.5, 0.0, 0.0],
                                  "children_left": [1, 0, 0], "children_right": [2, 0, 0],
                                  "default_left": [True, False, False],
                                  "leaf_values": {"type": "scalar", "values": [0.0, 1.0, 2.0]}}],
                       "n_groups": 1, "base_score": [0.25]},
            "output_transform": transform}


def envelope(model, version=2, kind="gbdt"):
    return json.dumps({"bstr_version": version, "model_type": kind, "model": model}).encode()


def zstd_frames(data, parts=1):
    """zstd frames from an independent encoder (pyarrow's bundled zstd), the
    data split into `parts` consecutive frames."""
    import pyarrow as pa
    cuts = [len(data) * i // parts for i in range(parts + 1)]
    return b"".join(pa.compress(data[a:b], codec="zstd", asbytes=True) for a, b in zip(cuts, cuts[1:]))


def binary(model, fmt=1, kind=1, version=2, payload=None, frames=1):
    if payload is None:
        payload = msgpack.packb(model, use_bin_type=True)
        if fmt == 2:
            payload = zstd_frames(payload, frames)
    head = b"BSTR" + struct.pack("<I", version) + bytes([fmt, kind]) + bytes(22)
    return head + payload + struct.pack("<QI", len(payload), crc32c(payload)) + bytes(4)


def tree0(m):
    return m.tree(0)


def binary_zstd(model):
    return binary(model, fmt=2)


def binary_zstd_two_frames(model):
    return binary(model, fmt=2, frames=2)


@pytest.mark.parametrize("encode", [envelope, binary, binary_zstd, binary_zstd_two_frames])
def test_read_stump(encode):
    m = bst.GBDTModel.from_bytes(encode(stump("sigmoid")))
    assert (m.n_trees, m.n_groups, m.n_features) == (1, 1, 2)
    t = tree0(m)
    np.testing.assert_array_equal(t["is_leaf"], [0, 1, 1])
    np.testing.assert_array_equal(t["left"][:1], [1])
    np.testing.assert_array_equal(t["right"][:1], [2])
    np.testing.assert_array_equal(t["threshold"][:1], np.float32([0.5]))
    np.testing.assert_array_equal(t["default_left"][:1], [1])
    np.testing.assert_array_equal(t["leaf_value"][1:], np.float32([1.0, 2.0]))


def test_json_round_trip_and_schema():
    m = bst.GBDTModel.from_bytes(envelope(stump("softmax" if False else "sigmoid")))
    doc = json.loads(m.to_json_bytes())
    assert doc["bstr_version"] == 2 and doc["model_type"] == "gbdt"
    model = doc["model"]
    assert model["output_transform"] == "sigmoid"
    assert model["meta"] == {"num_features": 2, "num_groups": 1}
    f = model["forest"]
    assert f["n_groups"] == 1 and f["base_score"] == [0.25] and "tree_groups" not in f
    t = f["trees"][0]
    assert t["num_nodes"] == 3 and t["children_left"] == [1, 0, 0] and t["children_right"] == [2, 0, 0]
    assert t["thresholds"][0] == 0.5 and t["default_left"] == [True, False, False]
    assert t["leaf_values"] == {"type": "scalar", "values": [0.0, 1.0, 2.0]}
    assert "categories" not in t  # skipped when empty (schema.rs:107-108)
    # pretty and compact documents describe the same model
    assert json.loads(m.to_json_bytes(pretty=True)) == doc
    again = bst.GBDTModel.from_bytes(m.to_json_bytes())
    assert json.loads(again.to_json_bytes()) == doc


def test_binary_payload_decodes_independently():
    import pyarrow as pa
    m = bst.GBDTModel.from_bytes(envelope(stump()))
    b = m.to_bytes(compression_level=0)
    assert b[:4] == b"BSTR" and struct.unpack("<I", b[4:8])[0] == 2 and b[8] == 1 and b[9] == 1
    assert b[10:32] == bytes(22)
    payload, trailer = b[32:-16], b[-16:]
    plen, crc = struct.unpack("<QI", trailer[:12])
    assert plen == len(payload) and crc == crc32c(payload) and trailer[12:] == bytes(4)
    doc = msgpack.unpackb(payload, raw=False)
    want = json.loads(m.to_json_bytes())["model"]
    assert doc == want
    assert bst.GBDTModel.from_bytes(b).to_bytes(compression_level=0) == b
    # the default is the reference's: zstd level 3 (format byte 0x02), whose
    # payload an independent decoder expands to the same MessagePack bytes
    z = m.to_bytes()
    assert z[8] == 2 and z[9] == 1
    zp, zt = z[32:-16], z[-16:]
    assert struct.unpack("<QI", zt[:12]) == (len(zp), crc32c(zp))
    assert pa.decompress(zp, decompressed_size=len(payload), codec="zstd", asbytes=True) == payload
    assert bst.GBDTModel.from_bytes(z).to_bytes() == z
    assert pickle.loads(pickle.dumps(m)).to_bytes() == z
    for level in (1, 19):
        assert bst.GBDTModel.from_bytes(m.to_bytes(compression_level=level)).to_json_bytes() == m.to_json_bytes()
    for level in (-1, 23):
        with pytest.raises(n.BoostersError) as e:
            m.to_bytes(compression_level=level)
        assert e.value.status == n.BST_ERR_INVALID_ARGUMENT


def test_categorical_and_groups():
    model = stump()
    model["meta"]["num_groups"] = model["forest"]["n_groups"] = 2
    model["forest"]["base_score"] = [0.0, 1.0]
    t2 = json.loads(json.dumps(model["forest"]["trees"][0]))
    t2["categories"] = {"node_indices": [0], "category_sets": [[1, 3, 33]]}
    model["forest"]["trees"].append(t2)
    model["forest"]["tree_groups"] = [0, 1]
    model["output_transform"] = "softmax"
    m = bst.GBDTModel.from_bytes(envelope(model))
    t = m.tree(1)
    assert t["split_type"][0] == 1 and t["group"] == 1
    np.testing.assert_array_equal(t["cat_words"], [(1 << 1) | (1 << 3), 1 << 1])
    doc = json.loads(m.to_json_bytes())["model"]
    assert doc["forest"]["tree_groups"] == [0, 1]
    assert doc["forest"]["trees"][1]["categories"] == {"node_indices": [0], "category_sets": [[1, 3, 33]]}
    assert bst.GBDTModel.from_bytes(m.to_bytes()).to_json_bytes() == m.to_json_bytes()


def test_unit_variant_forms_and_unknown_keys():
    model = stump()
    model["output_transform"] = {"sigmoid": None}  # an externally tagged unit variant
    model["meta"]["feature_names"] = ["a", "b"]
    model["forest"]["trees"][0]["gains"] = [1.5, 0.0, 0.0]
    m = bst.GBDTModel.from_bytes(binary(model))
    assert json.loads(m.to_json_bytes())["model"]["output_transform"] == "sigmoid"
    np.testing.assert_array_equal(m.tree(0)["gain"], np.float32([1.5, 0.0, 0.0]))


def _bad(model_bytes, match):
    with pytest.raises(n.BoostersError, match=match):
        bst.GBDTModel.from_bytes(model_bytes)


def test_rejections():
    _bad(b'{"bstr_version": 1, "model_type": "gbdt", "model": "not_an_object"}', "object")
    _bad(envelope(stump(), kind="gblinear"), "not gbdt")
    _bad(envelope(stump(), version=3), "version")
    m = stump()
    m["forest"]["trees"][0]["thresholds"] = [0.5]
    _bad(envelope(m), "length num_nodes")
    m = stump()
    m["forest"]["trees"][0]["children_right"] = [7, 0, 0]
    _bad(envelope(m), "out of range")
    m = stump()
    m["forest"]["trees"][0]["children_left"] = [1, 1, 0]
    m["forest"]["trees"][0]["children_right"] = [2, 2, 0]
    _bad(envelope(m), "cycle or a shared child")
    m = stump()
    m["forest"]["base_score"] = [0.0, 1.0]
    _bad(envelope(m), "base_score")
    m = stump()
    m["forest"]["trees"][0]["linear_coefficients"] = {"node_indices": [1], "coefficients": [[0.5]]}
    with pytest.raises(n.BoostersError) as e:
        bst.GBDTModel.from_bytes(envelope(m))
    assert e.value.status == n.BST_ERR_UNSUPPORTED
    good = binary(stump())
    corrupt = bytearray(good)
    corrupt[40] ^= 0xFF
    _bad(bytes(corrupt), "checksum")
    _bad(good[: len(good) // 2], "length|small|checksum")
    # a zstd payload that is not zstd (valid checksum): a decompression error
    _bad(binary(stump(), fmt=2, payload=b"\x28\xb5\x2f\xfd" + bytes(40)), "zstd")
    # a truncated zstd frame
    full = zstd_frames(msgpack.packb(stump(), use_bin_type=True))
    _bad(binary(stump(), fmt=2, payload=full[:-3]), "zstd")
    _bad(binary(stump(), fmt=0), "0x00")
    _bad(binary(stump(), kind=2), "not gbdt")


def test_files(tmp_path):
    m = bst.GBDTModel.from_bytes(envelope(stump()))
    for name in ("m.bstr", "m.bstr.json"):
        p = tmp_path / name
        m.save(p)
        raw = p.read_bytes()
        assert raw.startswith(b"BSTR") == (not name.endswith(".json"))
        assert bst.GBDTModel.load(p).to_json_bytes() == m.to_json_bytes()
    with pytest.raises(n.BoostersError, match="cannot open"):
        bst.GBDTModel.load(tmp_path / "missing.bstr")
