"""Reader and writer of FeNNol model files (``.fnx`` and ``.pkl``).

``FENNIX.save`` (``src/fennol/models/fennix.py:647-662``) writes the model
dictionary ``{cutoff, modules, preprocessing, energy_unit, energy_terms,
variables}`` with ``modules`` and ``preprocessing`` as lists of
``[name, params]`` pairs; ``FENNIX.load`` (``:664-690``) turns them back into
ordered dictionaries.  ``.pkl``/``.pickle`` files are Python pickles of that
dictionary; every other extension is Flax's msgpack encoding
(``flax.serialization.msgpack_serialize``; Flax is a third-party dependency of
the reference, version unpinned in its ``pyproject.toml``).

The msgpack encoding restated here is Flax's published format:

* a numpy array is the msgpack extension type 1 whose payload is the msgpack
  encoding of ``(shape, dtype name, C-order bytes)``;
* extension type 2 is a Python complex (payload: msgpack of ``(re, im)``),
  type 3 a numpy scalar (payload as for an array of shape ``()``);
* arrays above ``2**30 - 2**16`` bytes are stored as a dictionary
  ``{"__msgpack_chunked_array__": True, "shape": {"0": d0, ...},
  "chunks": {"0": flat_chunk0, ...}}`` and concatenated back on load;
* tuples are written as ``{"0": v0, "1": v1, ...}`` inside chunk records
  only; elsewhere the model dictionary holds lists.
"""

from __future__ import annotations

import pickle
from collections import OrderedDict
from pathlib import Path
from typing import Any, Dict

import msgpack
import numpy as np

EXT_NDARRAY, EXT_COMPLEX, EXT_NPSCALAR = 1, 2, 3
MAX_CHUNK_BYTES = 2 ** 30 - 2 ** 16
CHUNK_MARK = "__msgpack_chunked_array__"


def _array_payload(arr: np.ndarray) -> bytes:
    arr = np.asarray(arr, order="C")
    return msgpack.packb((list(arr.shape), arr.dtype.name, arr.tobytes("C")), use_bin_type=True)


def _array_from_payload(data: bytes) -> np.ndarray:
    shape, name, buf = msgpack.unpackb(data, raw=True)
    name = name.decode() if isinstance(name, bytes) else name
    if name == "bfloat16":
        raw = np.frombuffer(buf, dtype=np.uint16).astype(np.uint32) << 16
        return raw.view(np.float32).reshape(tuple(shape))
    return np.frombuffer(buf, dtype=np.dtype(name)).reshape(tuple(shape)).copy()


def _ext_pack(obj: Any):
    if isinstance(obj, np.ndarray):
        return msgpack.ExtType(EXT_NDARRAY, _array_payload(obj))
    if isinstance(obj, np.generic):
        return msgpack.ExtType(EXT_NPSCALAR, _array_payload(np.asarray(obj)))
    if isinstance(obj, complex):
        return msgpack.ExtType(EXT_COMPLEX, msgpack.packb((obj.real, obj.imag)))
    if isinstance(obj, tuple):
        return list(obj)
    if hasattr(obj, "detach"):  # torch tensor
        return msgpack.ExtType(EXT_NDARRAY, _array_payload(obj.detach().cpu().numpy()))
    raise TypeError(f"cannot serialise {type(obj).__name__}")


def _ext_unpack(code: int, data: bytes):
    if code == EXT_NDARRAY:
        return _array_from_payload(data)
    if code == EXT_NPSCALAR:
        return _array_from_payload(data)[()]
    if code == EXT_COMPLEX:
        re, im = msgpack.unpackb(data)
        return complex(re, im)
    return msgpack.ExtType(code, data)


def _chunk_large(tree: Any) -> Any:
    if isinstance(tree, dict):
        return {k: _chunk_large(v) for k, v in tree.items()}
    if isinstance(tree, (list, tuple)):
        return [_chunk_large(v) for v in tree]
    if isinstance(tree, np.ndarray) and tree.nbytes > MAX_CHUNK_BYTES:
        per = max(1, MAX_CHUNK_BYTES // tree.dtype.itemsize)
        flat = tree.reshape(-1)
        chunks = [flat[i:i + per] for i in range(0, flat.size, per)]
        return {CHUNK_MARK: True,
                "shape": {str(i): int(d) for i, d in enumerate(tree.shape)},
                "chunks": {str(i): c for i, c in enumerate(chunks)}}
    return tree


def _unchunk(tree: Any) -> Any:
    if isinstance(tree, dict):
        if tree.get(CHUNK_MARK, False):
            shape = tuple(tree["shape"][str(i)] for i in range(len(tree["shape"])))
            flat = np.concatenate([tree["chunks"][str(i)] for i in range(len(tree["chunks"]))])
            return flat.reshape(shape)
        return {k: _unchunk(v) for k, v in tree.items()}
    if isinstance(tree, list):
        return [_unchunk(v) for v in tree]
    return tree


def msgpack_serialize(tree: Dict[str, Any]) -> bytes:
    """Flax-compatible msgpack bytes of a tree of dicts, lists and arrays."""
    return msgpack.packb(_chunk_large(tree), default=_ext_pack, strict_types=True)


def msgpack_restore(data: bytes) -> Dict[str, Any]:
    """Inverse of :func:`msgpack_serialize`; arrays come back as numpy."""
    return _unchunk(msgpack.unpackb(data, ext_hook=_ext_unpack, raw=False))


def save_model_dict(state: Dict[str, Any], filename) -> None:
    """Write a model dictionary the way ``FENNIX.save`` does."""
    out = dict(state)
    out["preprocessing"] = [[k, v] for k, v in OrderedDict(state["preprocessing"]).items()]
    out["modules"] = [[k, v] for k, v in OrderedDict(state["modules"]).items()]
    name = str(filename)
    if name.endswith(".pkl") or name.endswith(".pickle"):
        with open(filename, "wb") as f:
            pickle.dump(_to_numpy(out), f)
    else:
        Path(filename).write_bytes(msgpack_serialize(out))


def load_model_dict(filename) -> Dict[str, Any]:
    """Read a model file written by ``FENNIX.save``; ``modules`` and
    ``preprocessing`` come back as ordered dictionaries."""
    name = str(filename)
    if name.endswith(".pkl") or name.endswith(".pickle"):
        with open(filename, "rb") as f:
            state = pickle.load(f)
    else:
        state = msgpack_restore(Path(filename).read_bytes())
    state["preprocessing"] = OrderedDict((k, v) for k, v in state["preprocessing"])
    state["modules"] = OrderedDict((k, v) for k, v in state["modules"])
    return state


def _to_numpy(tree: Any) -> Any:
    if isinstance(tree, dict):
        return {k: _to_numpy(v) for k, v in tree.items()}
    if isinstance(tree, (list, tuple)):
        return type(tree)(_to_numpy(v) for v in tree)
    if hasattr(tree, "detach"):
        return tree.detach().cpu().numpy()
    return tree
