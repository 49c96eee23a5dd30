"""dsss_distribute_lines (distribute_strings on one GPU) against the rank by
rank restatement of src/mpi/readInput.hpp:40-104: every PE's raw bytes (its
lines, each followed by a NUL), for line lengths from empty to longer than a
slice, files with and without a final newline, max_size, a NUL inside a line;
then the whole path on the distributed lines against the oracle."""
import numpy as np
import pytest

from test_gpu_parity import check_pd

pytestmark = pytest.mark.gpu


def text(seed, lines, maxlen, final_newline=True, nul=False):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(lines):
        m = int(rng.integers(0, maxlen + 1))
        out.append(bytes(rng.integers(97, 123, size=m, dtype=np.uint8)))
    if nul and out:
        out[len(out) // 2] = out[len(out) // 2] + b"\0x"
    data = b"\n".join(out)
    return data + b"\n" if final_newline else data


def per_pe(ds, pb):
    offs = ds.offsets[:ds.n].cpu().numpy() if ds.n else np.zeros(0, np.int64)
    lens = ds.lengths[:ds.n].cpu().numpy() if ds.n else np.zeros(0, np.int32)
    chars = ds.chars.cpu().numpy()
    out = []
    for r in range(len(pb) - 1):
        out.append(b"".join(chars[int(offs[k]):int(offs[k]) + int(lens[k])].tobytes() + b"\0"
                            for k in range(int(pb[r]), int(pb[r + 1]))))
    return out


CASES = [
    ("short", dict(seed=1, lines=3000, maxlen=12)),
    ("long", dict(seed=2, lines=400, maxlen=300)),
    ("no_final_newline", dict(seed=3, lines=2000, maxlen=20, final_newline=False)),
    ("nul_inside", dict(seed=4, lines=2000, maxlen=20, nul=True)),
]


@pytest.mark.parametrize("p", [1, 2, 5, 16])
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_distribute_matches_reference_rule(dsss, orc, ctx, name, kw, p):
    data = text(**kw)
    for max_size in (0, len(data) // 2 + 3):
        try:
            want = orc.distribute_strings(data, p, max_size)
        except ValueError:
            with pytest.raises(dsss.DsssError):
                dsss.distribute_lines(ctx, data, p, max_size)
            continue
        ds, pb = dsss.distribute_lines(ctx, data, p, max_size)
        assert per_pe(ds, pb) == want


def test_distribute_rejects_slice_without_newline(dsss, orc, ctx):
    data = b"a" * 5000 + b"\nb\n"
    with pytest.raises(ValueError):
        orc.distribute_strings(data, 4)
    with pytest.raises(dsss.DsssError):
        dsss.distribute_lines(ctx, data, 4)


@pytest.mark.parametrize("p", [3, 8])
def test_distributed_lines_through_the_path(dsss, orc, ctx, p):
    """The distributed lines as the sort's input: the oracle's full path on the
    same arena (the PE split is the distribution's)."""
    data = text(seed=9, lines=20000, maxlen=30)
    ds, pb = dsss.distribute_lines(ctx, data, p)
    out = dsss.pd_sort(ctx, ds, p, part_begin=pb)
    hs = dsss.from_bytes_list([bytes(x) for x in data.split(b"\n")[:-1]])
    assert hs.n == ds.n
    check_pd(dsss, orc, hs, out, p)


@pytest.mark.parametrize("data,p", [(b"", 1), (b"x", 1), (b"\n", 1), (b"a\nb\n", 2), (b"\n\n\n\n", 4),
                                    (b"ab\ncd", 2)])
def test_distribute_edges(dsss, orc, ctx, data, p):
    try:
        want = orc.distribute_strings(data, p)
    except ValueError:
        with pytest.raises(dsss.DsssError):
            dsss.distribute_lines(ctx, data, p)
        return
    ds, pb = dsss.distribute_lines(ctx, data, p)
    assert per_pe(ds, pb) == want
