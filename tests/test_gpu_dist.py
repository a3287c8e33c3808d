"""The slab decomposition (include/ops_b200_dist.h) on this backend: the
multi-block Poisson driver's single-block form split over 2 and 3 ranks,
every rank a process on the same GPU, rows exchanged through pinned host
memory and a gloo process group (no kernel of one rank waits on another's:
each exchange is a host step between launches).  Every dat, put back
together from the ranks' owned rows, equals the one-rank run bit for bit;
the max-residual reductions match exactly and the checksum (a sum combined
over the ranks in another order) to 1e-13."""

import pytest

from tests.apprun import ensure, result_lines, run_app
from tests.distrun import gather, run_ranks
from tests.opsdump import read_dump

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ranks,args", [(2, ["-nb=1", "-n=300", "-sweeps=60", "-check=20"]),
                                        (3, ["-nb=1", "-n=257", "-sweeps=45", "-check=15"])])
def test_b200_slab_decomposition_matches_one_rank(tmp_path, ranks, args):
    import numpy as np
    ensure("poisson_mb", "b200")
    one_out, one_dump = run_app("poisson_mb", "b200", args, dump=True)
    dump = str(tmp_path / "dist.dump")
    out = run_ranks("poisson_mb", "b200", args, ranks, dump)
    whole = read_dump(one_dump)
    parts = gather(dump, ranks)
    assert set(parts) == set(whole)
    for name, (meta, arr) in whole.items():
        assert np.array_equal(parts[name][1], arr), name
    res = [l for l in result_lines(out, ("sweep",))]
    assert res and res == [l for l in result_lines(one_out, ("sweep",))]
    c1 = float(result_lines(out, ("checksum",))[0].split()[1])
    c0 = float(result_lines(one_out, ("checksum",))[0].split()[1])
    assert abs(c1 - c0) <= 1e-13 * abs(c0)
