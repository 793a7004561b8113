"""Block streaming (src/core/stream.rs:650-1000) on the GPU: encode_stream,
verify_stream, reconstruct_stream and reconstruct_stream_from over file-like
objects, byte-exact against the oracle, with the reference's error rules."""
import io

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rs():
    import rsgpu

    return rsgpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    assert t.cuda.is_available()
    return t


def oracle_parity(codec, data):
    k, m = codec.data_shard_count(), codec.parity_shard_count()
    n = max(len(d) for d in data)
    sh = [np.frombuffer(d.ljust(n, b"\0"), np.uint8).copy() for d in data] + [np.zeros(n, np.uint8) for _ in range(m)]
    O.classic_encode(codec.encoding_matrix(), sh)
    return [bytes(s) for s in sh[k:]]


@pytest.mark.parametrize("k,m,length,block", [(10, 4, 3 * 1048576 + 777, 1 << 20), (4, 2, 5000, 1024),
                                              (6, 3, 100000, 0), (3, 2, 1 << 20, 64 << 20)])
def test_encode_stream_matches_oracle(rs, torch, k, m, length, block):
    c = rs.ReedSolomon(k, m)
    rng = np.random.default_rng(k * 100 + m)
    data = [rng.integers(0, 256, length, dtype=np.uint8).tobytes() for _ in range(k)]
    out = [io.BytesIO() for _ in range(m)]
    c.encode_stream([io.BytesIO(d) for d in data], out, block_size=block)
    want = oracle_parity(c, data)
    for r in range(m):
        assert out[r].getvalue() == want[r], r


def test_encode_stream_zero_pads_shorter_streams(rs, torch):
    c = rs.ReedSolomon(4, 2)
    rng = np.random.default_rng(3)
    lens = [3000, 2500, 3000, 1]
    data = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for n in lens]
    out = [io.BytesIO() for _ in range(2)]
    c.encode_stream([io.BytesIO(d) for d in data], out, block_size=1024)
    want = oracle_parity(c, data)
    assert [o.getvalue() for o in out] == want
    # an all-empty input writes nothing
    out = [io.BytesIO() for _ in range(2)]
    c.encode_stream([io.BytesIO(b"") for _ in range(4)], out)
    assert all(o.getvalue() == b"" for o in out)


def test_verify_stream(rs, torch):
    k, m, n = 5, 3, 70000
    c = rs.ReedSolomon(k, m)
    rng = np.random.default_rng(9)
    data = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for _ in range(k)]
    full = data + oracle_parity(c, data)
    assert c.verify_stream([io.BytesIO(s) for s in full], block_size=4096)
    bad = list(full)
    b = bytearray(bad[k + 1])
    b[5 * 4096 + 17] ^= 0x40
    bad[k + 1] = bytes(b)
    assert not c.verify_stream([io.BytesIO(s) for s in bad], block_size=4096)
    short = list(full)
    short[2] = short[2][:-1]
    with pytest.raises(rs.StreamError) as e:
        c.verify_stream([io.BytesIO(s) for s in short], block_size=4096)
    assert e.value.kind == "codec" and e.value.shard_index == 2 and e.value.error.name == "IncorrectShardSize"


@pytest.mark.parametrize("lost", [[0], [1, 6], [0, 2, 5], [7, 6, 5]])
def test_reconstruct_stream_matches_oracle(rs, torch, lost):
    k, m, n = 5, 3, 300001
    c = rs.ReedSolomon(k, m)
    rng = np.random.default_rng(len(lost))
    data = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for _ in range(k)]
    full = data + oracle_parity(c, data)
    cur = [io.BytesIO(b"" if i in lost else full[i]) for i in range(k + m)]
    for i in range(k + m):
        if i not in lost:
            cur[i].seek(0, io.SEEK_END)  # positions are reset by reconstruct_stream
    c.reconstruct_stream(cur, block_size=65536)
    for i in range(k + m):
        assert cur[i].getvalue() == full[i], i
    # reconstruct_stream_from with separate readers and writers
    writers = [io.BytesIO() if i in lost else None for i in range(k + m)]
    readers = [None if i in lost else io.BytesIO(full[i]) for i in range(k + m)]
    c.reconstruct_stream_from(readers, writers, block_size=100000)
    for i in lost:
        assert writers[i].getvalue() == full[i]


def test_reconstruct_stream_on_non_codewords_matches_oracle(rs, torch):
    k, m, n = 4, 2, 9000
    c = rs.ReedSolomon(k, m)
    rng = np.random.default_rng(1)
    shards = [rng.integers(0, 256, n, dtype=np.uint8) for _ in range(k + m)]
    present = [0, 1, 1, 1, 0, 1]
    ref = [s.copy() for s in shards]
    ref[0][:] = 0
    ref[4][:] = 0
    assert O.classic_reconstruct(c.encoding_matrix(), ref, present) == 0
    cur = [io.BytesIO(b"" if not present[i] else shards[i].tobytes()) for i in range(k + m)]
    c.reconstruct_stream(cur, block_size=2048)
    for i in range(k + m):
        assert cur[i].getvalue() == ref[i].tobytes(), i


def test_stream_errors(rs, torch):
    c = rs.ReedSolomon(4, 2)
    with pytest.raises(rs.StreamError) as e:
        c.encode_stream([io.BytesIO(b"x")] * 3, [io.BytesIO(), io.BytesIO()])
    assert e.value.error.name == "TooFewShards"
    with pytest.raises(rs.StreamError) as e:
        c.encode_stream([io.BytesIO(b"x")] * 4, [io.BytesIO()] * 3)
    assert e.value.error.name == "TooManyShards"
    leo = rs.ReedSolomon(4, 2, rs.CodecOptions(codec_family="leopard_gf8"))
    with pytest.raises(rs.StreamError) as e:
        leo.encode_stream([io.BytesIO(b"x" * 64)] * 4, [io.BytesIO()] * 2)
    assert e.value.error.name == "UnsupportedCodecFamily"
    with pytest.raises(rs.StreamError) as e:
        leo.verify_stream([io.BytesIO(b"x" * 64)] * 6)
    assert e.value.error.name == "UnsupportedCodecFamily"
    # reader and writer on the same index -> InvalidShardFlags with that index
    readers = [io.BytesIO(b"a" * 10) for _ in range(6)]
    writers = [None] * 6
    writers[3] = io.BytesIO()
    with pytest.raises(rs.StreamError) as e:
        c.reconstruct_stream_from(readers, writers)
    assert e.value.error.name == "InvalidShardFlags" and e.value.shard_index == 3
    readers = [None, None, None, io.BytesIO(b"a"), io.BytesIO(b"a"), io.BytesIO(b"a")]
    writers = [io.BytesIO(), io.BytesIO(), io.BytesIO(), None, None, None]
    with pytest.raises(rs.StreamError) as e:
        c.reconstruct_stream_from(readers, writers)
    assert e.value.error.name == "TooFewShardsPresent"
    # unequal present lengths -> IncorrectShardSize at the first short one
    readers = [None, io.BytesIO(b"a" * 100), io.BytesIO(b"a" * 99), io.BytesIO(b"a" * 100), io.BytesIO(b"a" * 100),
               io.BytesIO(b"a" * 100)]
    writers = [io.BytesIO(), None, None, None, None, None]
    with pytest.raises(rs.StreamError) as e:
        c.reconstruct_stream_from(readers, writers)
    assert e.value.error.name == "IncorrectShardSize" and e.value.shard_index == 2


class FailingReader(io.RawIOBase):
    def __init__(self, data, fail_at):
        self.b = io.BytesIO(data)
        self.fail_at = fail_at

    def readable(self):
        return True

    def readinto(self, buf):
        if self.b.tell() >= self.fail_at:
            raise OSError("disk went away")
        return self.b.readinto(buf)


def test_read_error_keeps_written_prefix(rs, torch):
    k, m, n, block = 4, 2, 10 * 1024, 1024
    c = rs.ReedSolomon(k, m)
    rng = np.random.default_rng(2)
    data = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for _ in range(k)]
    readers = [io.BytesIO(d) for d in data]
    readers[2] = FailingReader(data[2], 4 * block)
    out = [io.BytesIO() for _ in range(m)]
    with pytest.raises(rs.StreamError) as e:
        c.encode_stream(readers, out, block_size=block)
    assert e.value.kind == "read" and e.value.shard_index == 2 and isinstance(e.value.error, OSError)
    want = oracle_parity(c, [d[: 4 * block] for d in data])
    assert [o.getvalue() for o in out] == want  # the four blocks before the failure
