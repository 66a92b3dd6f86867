"""The Python API's sequence arguments for the C ABI (pointer and length
arrays over one joined buffer): every pointer addresses its sequence's bytes,
empty sequences and empty lists included. No GPU needed."""
import ctypes

import numpy as np

from minipoa_b200.api import _seq_arrays


def test_pointer_and_length_arrays_address_every_sequence():
    rng = np.random.default_rng(7)
    seqs = [bytes(rng.integers(65, 91, size=int(n), dtype=np.uint8)) for n in rng.integers(0, 300, size=500)]
    seqs[3] = b""
    seqs.append(bytearray(b"ACGT"))  # bytes-like inputs are accepted too
    arr, lens, keep = _seq_arrays(seqs)
    for i, s in enumerate(seqs):
        assert lens[i] == len(s)
        assert ctypes.string_at(arr[i], len(s)) == bytes(s)
    # consecutive sequences are laid out back to back
    assert ctypes.addressof(arr[1].contents) - ctypes.addressof(arr[0].contents) == len(seqs[0])


def test_empty_inputs():
    arr, lens, keep = _seq_arrays([])
    assert lens[0] == 0
    arr, lens, keep = _seq_arrays([b"", b"", b"A"])
    assert [lens[i] for i in range(3)] == [0, 0, 1]
    assert ctypes.string_at(arr[2], 1) == b"A"
