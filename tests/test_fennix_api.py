"""Host-side behaviour of the FeNNol-compatible API (no GPU): construction
from FeNNol model dictionaries, model files, the species indexer and the
overflow protocol."""

import dataclasses
import pickle
from collections import OrderedDict

import msgpack
import numpy as np
import pytest

from fennol_b200 import fnx
from fennol_b200.fennix import (FENNIX, PREPROCESSING, SpeciesIndexer, energy_multiplier,
                                parse_celu, register_preprocessing)

SPECIES7 = ["H", "C", "N", "O", "S", "F", "Cl"]


def ani_modules(species=SPECIES7, activation="partial(celu,alpha=0.1)", hidden=(256, 192, 160)):
    return OrderedDict(
        embedding=dict(module_name="ANI_AEV", species_order=list(species), graph_angle_key="graph_angle",
                       radial_eta=19.7, angular_eta=12.5, radial_dist_divisions=16,
                       angular_dist_divisions=8, zeta=14.1, angle_sections=4, radial_start=0.9,
                       angular_start=0.9),
        energy=dict(module_name="SPECIES_INDEX_NET", species_order=list(species), activation=activation,
                    output_dim=1, hidden_neurons=list(hidden), input_key="embedding", squeeze=True))


def ani_preprocessing():
    return OrderedDict(
        graph_filter_angle=dict(module_name="GRAPH_FILTER", cutoff=3.5, graph_key="graph_angle",
                                parent_graph="graph"),
        angle_extension=dict(module_name="GRAPH_ANGULAR_EXTENSION", graph_key="graph_angle"),
        species_indexer=dict(output_key="species_index"))


def test_build_from_fennol_dicts():
    m = FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"])
    assert m.aev_config.aev_length == 1008
    assert m.aev_config.radial_cutoff == 5.2 and m.aev_config.angular_cutoff == 3.5
    assert m.mlp_config.hidden == (256, 192, 160) and m.mlp_config.celu_alpha == 0.1
    assert [type(l).__name__ for l in m.preprocessing.layers] == [
        "GraphGenerator", "GraphFilter", "GraphAngularExtension", "SpeciesIndexer"]
    props = m.preprocessing.get_graphs_properties()
    assert props["graph"]["cutoff"] == 5.2 and props["graph_angle"]["parent_graph"] == "graph"
    kernel = m.variables["params"]["energy"]["H"]["Layer_1"]["kernel"]
    assert kernel.shape == (1008, 256)


def test_reference_example_species_subset():
    """The reference's training example uses H, C, N, O with cutoff 5.1."""
    m = FENNIX(5.1, ani_modules(species=["H", "C", "N", "O"]), ani_preprocessing(),
               energy_terms=["energy"])
    assert m.aev_config.aev_length == 4 * 16 + 10 * 32


def test_unsupported_parts_raise():
    mods = ani_modules()
    mods["repulsion"] = dict(module_name="REPULSION_ZBL", trainable=True)
    with pytest.raises(NotImplementedError):
        FENNIX(5.2, mods, ani_preprocessing())
    with pytest.raises(NotImplementedError):
        FENNIX(5.2, ani_modules(activation="silu"), ani_preprocessing())
    with pytest.raises(NotImplementedError):
        FENNIX(5.2, ani_modules(hidden=(64, 64)), ani_preprocessing())
    with pytest.raises(NotImplementedError):
        FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy", "repulsion"])
    with pytest.raises(NotImplementedError):
        FENNIX(5.2, ani_modules(), OrderedDict(graph=dict(switch_params={"switch_type": "polynomial"})))


@pytest.mark.parametrize("suffix", [".fnx", ".pkl"])
def test_save_load_round_trip(tmp_path, suffix):
    m = FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"], rng_key=3)
    path = tmp_path / f"model{suffix}"
    m.save(path)
    m2 = FENNIX.load(path)
    assert m2.aev_config == m.aev_config and m2.mlp_config == m.mlp_config
    assert m2.energy_terms == ["energy"] and m2.cutoff == 5.2
    for sym in SPECIES7:
        for k in range(1, 5):
            a = m.variables["params"]["energy"][sym][f"Layer_{k}"]
            b = m2.variables["params"]["energy"][sym][f"Layer_{k}"]
            np.testing.assert_array_equal(a["kernel"], b["kernel"])
            np.testing.assert_array_equal(a["bias"], b["bias"])


def test_msgpack_layout_matches_flax_format():
    arr = np.arange(12, dtype=np.float32).reshape(3, 4)
    blob = fnx.msgpack_serialize({"a": arr, "s": np.float64(1.5), "l": [1, "x"]})
    raw = msgpack.unpackb(blob, raw=False, ext_hook=lambda c, d: (c, d))
    code, payload = raw["a"]
    assert code == fnx.EXT_NDARRAY
    shape, dtype, data = msgpack.unpackb(payload, raw=True)
    assert list(shape) == [3, 4] and dtype == b"float32" and data == arr.tobytes()
    assert raw["s"][0] == fnx.EXT_NPSCALAR
    back = fnx.msgpack_restore(blob)
    np.testing.assert_array_equal(back["a"], arr)
    assert back["s"] == 1.5 and back["l"] == [1, "x"]


def test_msgpack_chunked_and_bfloat16_records():
    flat = np.arange(10, dtype=np.float64)
    rec = {fnx.CHUNK_MARK: True, "shape": {"0": 2, "1": 5},
           "chunks": {"0": flat[:6], "1": flat[6:]}}
    blob = fnx.msgpack_serialize({"w": rec})
    np.testing.assert_array_equal(fnx.msgpack_restore(blob)["w"], flat.reshape(2, 5))
    vals = np.array([1.0, -2.5, 0.15625], np.float32)
    bits = (vals.view(np.uint32) >> 16).astype(np.uint16)
    payload = msgpack.packb(([3], "bfloat16", bits.tobytes()), use_bin_type=True)
    blob = msgpack.packb({"b": msgpack.ExtType(fnx.EXT_NDARRAY, payload)})
    np.testing.assert_array_equal(fnx.msgpack_restore(blob)["b"], vals)


def test_species_indexer_dict_and_dense():
    sp = np.array([8, 1, 1, 8, 1, 1, 6], np.int32)
    layer = SpeciesIndexer()
    state, out = layer(layer.init(), {"species": sp})
    idx = out["species_index"]
    np.testing.assert_array_equal(idx["O"], [0, 3])
    np.testing.assert_array_equal(idx["H"], [1, 2, 4, 5])
    np.testing.assert_array_equal(idx["C"], [6])
    assert state["sizes"] == {1: 4, 6: 1, 8: 2}
    dense = SpeciesIndexer(species_order="H,C,O", add_atoms=1)
    state, out = dense(dense.init(), {"species": sp})
    d = out["species_index"]
    assert d.shape == (3, 5)
    np.testing.assert_array_equal(d[0], [1, 2, 4, 5, 7])
    np.testing.assert_array_equal(d[2], [0, 3, 7, 7, 7])


def test_species_indexer_overflow_protocol():
    layer = SpeciesIndexer()
    state, _ = layer(layer.init(), {"species": np.array([1, 1, 8])})
    more = {"species": np.array([1, 1, 1, 8])}
    out = layer.process(state, more)
    assert out["species_index_overflow"]
    state2, up, out2, realloc = layer.check_reallocate(state, out)
    assert realloc and up["sizes"][0][1] == 3 + layer.add_atoms_margin
    np.testing.assert_array_equal(out2["species_index"]["H"][:3], [0, 1, 2])
    _, up3, _, realloc3 = layer.check_reallocate(state2, layer.process(state2, more))
    assert not realloc3 and up3 == {}


def test_external_preprocessing_registration():
    @register_preprocessing
    @dataclasses.dataclass(frozen=True)
    class Tagger:
        tag: str = "x"
        FPID = "TEST_TAGGER"

        def init(self):
            return {}

        def __call__(self, state, inputs, return_state_update=False, add_margin=False):
            out = {**inputs, "tag": self.tag}
            return (state, out, {}) if return_state_update else (state, out)

    try:
        prep = ani_preprocessing()
        prep["tagger"] = dict(module_name="TEST_TAGGER", tag="y")
        m = FENNIX(5.2, ani_modules(), prep, energy_terms=["energy"])
        assert type(m.preprocessing.layers[-1]).__name__ == "Tagger"
        assert m.preprocessing.layers[-1].tag == "y"
    finally:
        PREPROCESSING.pop("TEST_TAGGER", None)


def test_activation_and_units():
    assert parse_celu("partial(celu,alpha=0.1)") == 0.1
    assert parse_celu("celu") == 1.0 and parse_celu("jax.nn.celu") == 1.0
    with pytest.raises(NotImplementedError):
        parse_celu("silu")
    assert energy_multiplier("kcalpermol") == pytest.approx(627.5096080305927)
    assert energy_multiplier("eV") == pytest.approx(27.211386024367243)
    m = FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"],
               energy_unit="kcalpermol")
    assert m._unit_factor("Ha") == pytest.approx(1 / 627.5096080305927)


def test_overflow_flag_reads_its_words_when_tested():
    """A graph layer's overflow entry: false until one of its status words is
    set, read from the (here host) status tensor only when tested."""
    import torch

    from fennol_b200 import _lib
    from fennol_b200.fennix import OverflowFlag

    status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32)
    flag = OverflowFlag(status, (_lib.ST_NBR_OVERFLOW, _lib.ST_FILTER_OVERFLOW))
    assert not flag and flag.item() is False
    status[_lib.ST_FILTER_OVERFLOW] = 1
    assert flag and "True" in repr(flag)
    status.zero_()
    status[_lib.ST_NBR_MAXCOUNT] = 40  # other words do not count
    assert not flag
