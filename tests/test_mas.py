"""MAS checkpoint format (PSuM's src/serialization/mas.hpp) on the host."""
import struct

import numpy as np
import pytest

import psum_b200 as P
from psum_b200 import mas


def test_block_byte_layout(tmp_path):
    # mas_file::writeData (mas.hpp:130-152): magic, three int32 lengths, key,
    # type name, uint64 shape, then the elements
    fp = mas.MasFile(tmp_path / "a.mas", "replace")
    fp.write("data1", np.arange(4, dtype=np.float64))
    expect = (b"#MAS!#" + struct.pack("<iii", 5, 6, 2) + b"data1" + b"double" + struct.pack("<2Q", 4, 1)
              + np.arange(4, dtype="<f8").tobytes())
    assert (tmp_path / "a.mas").read_bytes() == expect


def test_types_round_trip(tmp_path):
    path = tmp_path / "t.mas"
    fp = mas.MasFile(path, "replace")
    arrays = {
        "d": np.linspace(0, 1, 7), "f": np.arange(5, dtype=np.float32),
        "i64": np.arange(-3, 3, dtype=np.int64), "u64": np.arange(3, dtype=np.uint64),
        "i32": np.arange(6, dtype=np.int32).reshape(2, 3), "u32": np.array([7], np.uint32),
        "i16": np.array([-2, 2], np.int16), "u16": np.array([9], np.uint16),
        "i8": np.array([-1], np.int8), "u8": np.array([255], np.uint8), "b": np.array([True, False]),
    }
    for k, v in arrays.items():
        fp.write(k, v)
    fp.write("s", "[#0]NVIDIA B200")
    fp.write("scalar", np.array([3], np.int32), (1, 1))
    again = mas.MasFile(path)       # auto mode reads the heads
    assert again.keys() == list(arrays) + ["s", "scalar"]
    for k, v in arrays.items():
        h, got = again.read(k)
        assert got.dtype == v.dtype
        assert (got.reshape(-1) == v.reshape(-1)).all()
        assert h.shape == ((v.size, 1) if v.ndim == 1 else v.shape)
    assert again.read_string("s") == "[#0]NVIDIA B200"
    assert [h.type for h in again.heads][:3] == ["double", "single", "int64"]


def test_reference_basic_flow(tmp_path):
    # the flow of PSuM's test/serialization/test_mas.cpp: three arrays
    # written, read back, one replaced and read again
    fp = mas.MasFile(tmp_path / "test.mas")
    fp.clear()
    n = 100
    fp.write("data1", np.arange(n, dtype=np.float64), (n, 1))
    fp.write("data2", np.arange(n, dtype=np.int32), (n, 1))
    fp.write("data3", np.arange(n, dtype=np.float32), (n, 1))
    fp.read_head()
    assert (fp.read("data1")[1].reshape(-1) == np.arange(n)).all()
    assert (fp.read("data2")[1].reshape(-1) == np.arange(n)).all()
    assert (fp.read("data3")[1].reshape(-1) == np.arange(n)).all()
    fp.read_head()
    fp.replace("data1", 2.0 * np.arange(n), (n, 1))
    fp.read_head()
    assert (fp.read("data1")[1].reshape(-1) == 2 * np.arange(n)).all()
    assert fp.keys() == ["data2", "data3", "data1"]   # the old block is masked, not removed


def test_mask_duplicate_and_errors(tmp_path):
    path = tmp_path / "m.mas"
    fp = mas.MasFile(path, "replace")
    fp.write("x", np.ones(3))
    with pytest.raises(mas.MasDuplicateBlockError):
        fp.write("x", np.zeros(2, np.int32))          # any type: strict name checking
    with pytest.raises(ValueError):
        fp.write("!x", np.ones(1))
    with pytest.raises(ValueError):
        fp.write("", np.ones(1))
    assert fp.smash("x")
    assert mas.MasFile(path).keys() == []
    raw = path.read_bytes()
    assert raw[6 + 12:6 + 13] == b"!"                  # '!' over the key's first byte
    fp.write("x", np.zeros(2))                          # the key is free again
    assert (mas.MasFile(path).read("x")[1].reshape(-1) == 0).all()
    with pytest.raises(FileNotFoundError):
        mas.MasFile(tmp_path / "missing.mas", "quick")
    (tmp_path / "bad.mas").write_bytes(b"#MAX!#" + bytes(12))
    with pytest.raises(ValueError):
        mas.MasFile(tmp_path / "bad.mas")


def test_grid_and_node_field(tmp_path):
    g = P.simple_grid((0.0, -1.0), (4.0, 1.0), (8, 4))
    phi = np.random.default_rng(1).normal(size=g.n_nodes)
    fp = mas.MasFile(tmp_path / "f.mas", "replace")
    mas.save_node_field(fp, "phi", g, phi)
    fp2 = mas.MasFile(tmp_path / "f.mas")
    assert fp2.keys() == ["phi.location", "phi.grid.lower", "phi.grid.upper", "phi.grid.cells",
                          "phi.content.device", "phi.content.content"]
    assert fp2.read("phi.location")[0].type == "int32"
    lower, upper, cells = mas.load_grid(fp2, "phi.grid")
    assert list(lower) == [0.0, -1.0] and list(upper) == [4.0, 1.0] and list(cells) == [8, 4]
    got = mas.load_node_field(fp2, "phi", g)
    assert (got.view(np.int64) == phi.view(np.int64)).all()
    with pytest.raises(ValueError):
        mas.load_node_field(fp2, "phi", P.simple_grid((0.0, -1.0), (4.0, 1.0), (8, 5)))


def test_random_block_sequences_round_trip(tmp_path):
    # hypothesis: random sequences of blocks of every element type and shape
    # (empty ones included), written, reopened, partly masked with smash and
    # read back (mas.hpp:130-330)
    from hypothesis import HealthCheck, given, settings, strategies as st
    import hypothesis.extra.numpy as hnp

    dtypes = [np.float64, np.float32, np.int64, np.uint64, np.int32, np.uint32, np.int16, np.uint16, np.int8,
              np.uint8, np.bool_]
    block = st.tuples(st.sampled_from(dtypes), hnp.array_shapes(min_dims=1, max_dims=3, min_side=0, max_side=5))
    counter = iter(range(10 ** 9))

    @settings(max_examples=40, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(st.lists(block, min_size=1, max_size=8), st.data())
    def check(blocks, data):
        path = tmp_path / f"r{next(counter)}.mas"
        fp = mas.MasFile(path, "replace")
        written = {}
        for i, (dt, shape) in enumerate(blocks):
            arr = data.draw(hnp.arrays(dt, shape, elements=hnp.from_dtype(np.dtype(dt), allow_nan=False)))
            key = f"b{i}.{np.dtype(dt).name}"
            fp.write(key, arr, shape)
            written[key] = arr
        with pytest.raises(mas.MasDuplicateBlockError):
            fp.write(next(iter(written)), np.zeros(1))
        masked = {k for k in written if data.draw(st.booleans())}
        again = mas.MasFile(path)
        for k in masked:
            assert again.smash(k)
        reread = mas.MasFile(path)
        assert reread.keys() == [k for k in written if k not in masked]
        for k, arr in written.items():
            h, got = reread.read(k)
            if k in masked:
                assert h is None
                continue
            assert h.shape == tuple(arr.shape) and got.dtype == arr.dtype
            assert (got == arr).all()

    check()
