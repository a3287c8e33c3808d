"""GPU tests of lazy execution: the loop-chain queue, its tiled execution and
its CUDA-graph replay give results bit-identical to eager execution.

Tiled execution runs every point through the same kernel as eager execution,
only split into skewed row tiles, so every dat must match exactly (max
difference 0).  Small forced tile heights (OPS_B200_TILESIZE_Y/Z) make many
tiles per chain, so the skew of every dependency pair is exercised.
"""

import os
import re
import subprocess
import sys

import pytest

from tests.apprun import ROOT, ensure, result_lines, run_app
from tests.opsdump import compare

pytestmark = pytest.mark.gpu

EAGER = {"OPS_B200_LAZY": "0", "OPS_B200_TILING": "0"}
MODES = {
    "lazy_graphs": {"OPS_B200_LAZY": "1", "OPS_B200_TILING": "0", "OPS_B200_GRAPHS": "1"},
    "lazy_single": {"OPS_B200_LAZY": "1", "OPS_B200_MULTI": "0", "OPS_B200_GRAPHS": "0"},
    "tiled_plain": {"OPS_B200_TILING": "1", "OPS_B200_GRAPHS": "0", "OPS_B200_TILESIZE_Y": "7",
                    "OPS_B200_TILESIZE_Z": "3"},
    "tiled_graphs": {"OPS_B200_TILING": "1", "OPS_B200_GRAPHS": "1", "OPS_B200_TILESIZE_Y": "5",
                     "OPS_B200_TILESIZE_Z": "2"},
    "tiled_cache": {"OPS_B200_TILING": "1", "OPS_B200_GRAPHS": "1", "OPS_B200_CACHE_MB": "0.25"},
}


def numbers_only(lines):
    """result lines without their timing fields"""
    return [re.sub(r"\S+ ms/step|\S+ s\b|\S+ GLUPS", "", l) for l in lines]


def same(a, b):
    d = compare(a, b)
    bad = {k: v for k, v in d.items() if v != 0.0}
    assert not bad, bad


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("app,args", [
    ("poisson_mb", ["-nb=1", "-n=200", "-sweeps=40", "-check=10"]),
    ("poisson_mb", ["-nb=3", "-n=61", "-sweeps=25", "-check=5"]),
    ("opsunit", ["-nx=45", "-ny=38"]),
    ("adi3d", ["-nx=40", "-ny=23", "-nz=17", "-steps=3", "-prec=64"]),
])
def test_lazy_matches_eager(app, args, mode):
    eo, ed = run_app(app, "b200", args, dump=True, env=EAGER)
    lo, ld = run_app(app, "b200", args, dump=True, env=MODES[mode])
    same(ld, ed)
    assert numbers_only(result_lines(lo)) == numbers_only(result_lines(eo))


@pytest.mark.parametrize("args", [["-nb=2", "-n=61", "-sweeps=25", "-check=5"],
                                  ["-nb=2", "-n=256", "-sweeps=40", "-check=10"]])
def test_halo_transfers_fold_into_the_consuming_launch(args):
    """The multi-block Jacobi: every sweep's ops_halo_transfer is folded into
    the launch of the four blocks' Jacobi loop (each CTA copies the halo
    cells its stencil reads, then computes); every dat equals eager
    execution bit for bit, and the same with folding switched off."""
    eo, ed = run_app("poisson_mb", "b200", args, dump=True, env=EAGER)
    lo, ld = run_app("poisson_mb", "b200", args, dump=True,
                     env={"OPS_B200_LAZY": "1", "OPS_B200_HFUSE": "1"})
    no, nd = run_app("poisson_mb", "b200", args, dump=True,
                     env={"OPS_B200_LAZY": "1", "OPS_B200_HFUSE": "0"})
    sweeps = int(args[2].split("=")[1])
    folded = int(re.search(r"(\d+) halo transfers folded", lo).group(1))
    assert folded >= sweeps - sweeps // int(args[3].split("=")[1])
    assert int(re.search(r"(\d+) halo transfers folded", no).group(1)) == 0
    same(ld, ed)
    same(nd, ed)
    assert numbers_only(result_lines(lo)) == numbers_only(result_lines(eo))


@pytest.mark.parametrize("depth,args", [
    ("2", ["-nb=1", "-n=203", "-sweeps=37", "-check=0"]),
    ("3", ["-nb=1", "-n=130", "-sweeps=20", "-check=5"]),
    ("8", ["-nb=1", "-n=257", "-sweeps=45", "-check=0"]),
    ("8", ["-nb=1", "-n=64", "-sweeps=130", "-check=0"])])
def test_temporal_blocking_matches_eager(depth, args):
    """Single-block Jacobi: the queued sweeps ping-pong u and u2, so they run
    temporally blocked (`depth` sweeps per launch in shared memory, u's
    storage moving to its spare buffer at every launch); every dat and every
    printed residual equal eager execution bit for bit (ragged sizes: edge
    tiles; odd chain lengths: a last sweep on its own; chains longer than 64
    items: flushes inside the run)."""
    eo, ed = run_app("poisson_mb", "b200", args, dump=True, env=EAGER)
    lo, ld = run_app("poisson_mb", "b200", args, dump=True,
                     env={"OPS_B200_LAZY": "1", "OPS_B200_TB": "1", "OPS_B200_TB_DEPTH": depth})
    m = re.search(r"(\d+) temporal-blocking launches \((\d+) sweeps\)", lo)
    assert m and int(m.group(1)) > 0 and int(m.group(2)) >= int(m.group(1)) * 2, lo[-600:]
    same(ld, ed)
    assert numbers_only(result_lines(lo)) == numbers_only(result_lines(eo))


def test_temporal_blocking_depth_autotuned():
    """OPS_B200_TB_DEPTH=auto: the first chains of the Jacobi sweeps run with
    each candidate depth (1 = plain sweeps, 2, 4, 8) outside graphs and timed,
    then one depth is kept; every dat and printed residual still equal eager
    execution bit for bit, and the run reports the depth it chose."""
    args = ["-nb=1", "-n=257", "-sweeps=1100", "-check=0"]
    eo, ed = run_app("poisson_mb", "b200", args, dump=True, env=EAGER)
    lo, ld = run_app("poisson_mb", "b200", args, dump=True,
                     env={"OPS_B200_LAZY": "1", "OPS_B200_TB": "1", "OPS_B200_TB_DEPTH": "auto"})
    m = re.search(r"Temporal-blocking depths \(1: plain sweeps\):((?: \S+=\d+)+)", lo)
    assert m, lo[-800:]
    depths = [int(x.split("=")[1]) for x in m.group(1).split()]
    assert depths and all(d in (1, 2, 4, 8) for d in depths), m.group(0)
    same(ld, ed)
    assert numbers_only(result_lines(lo)) == numbers_only(result_lines(eo))


@pytest.mark.parametrize("mode", ["lazy_graphs", "tiled_graphs", "tiled_cache"])
def test_cloverleaf_lazy_matches_eager(tmp_path, mode):
    ensure("clover_step", "b200")
    dumps = {}
    for tag, env in (("eager", EAGER), (mode, MODES[mode])):
        dumps[tag] = str(tmp_path / ("%s.dump" % tag))
        r = subprocess.run([sys.executable, "-m", "apps.clover_run", "--flavour", "b200",
                            "--cells", "120", "--steps", "12", "--dump", dumps[tag]], cwd=ROOT,
                           env=dict(os.environ, **env), capture_output=True, text=True,
                           timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
    same(dumps[mode], dumps["eager"])


def test_mblock_halos_lazy_matches_eager(tmp_path):
    """Queued ops_halo_transfer groups (multi-block, permuted and flipped)."""
    exe = ensure("ref_mblock", "b200", shared=False)
    dumps = {}
    for tag, env in (("eager", EAGER), ("lazy", MODES["tiled_graphs"])):
        dumps[tag] = str(tmp_path / ("%s.dump" % tag))
        r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True,
                           env=dict(os.environ, OPS_DUMP_FILE=dumps[tag], **env), timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
    same(dumps["lazy"], dumps["eager"])


AUTOTUNE = {"OPS_B200_AUTOTUNE": "1"}


@pytest.mark.parametrize("app,args", [
    ("poisson_mb", ["-nb=3", "-n=61", "-sweeps=25", "-check=5"]),
    ("opsunit", ["-nx=45", "-ny=38"]),
    ("adi3d", ["-nx=40", "-ny=23", "-nz=17", "-steps=3", "-prec=64"]),
])
def test_autotuned_block_shapes_give_identical_results(app, args):
    """The block-shape autotuner launches each candidate shape once and keeps
    the fastest; loops without reductions compute every point the same way
    under any shape (loops with reductions are not tuned), so every dat is
    bit-identical to the default shape's run."""
    eo, ed = run_app(app, "b200", args, dump=True, env=EAGER)
    to, td = run_app(app, "b200", args + ["-OPS_DIAGS=1"], dump=True, env=AUTOTUNE)
    same(td, ed)
    assert numbers_only(result_lines(to)) == numbers_only(result_lines(eo))


def test_cloverleaf_autotuned_matches_default(tmp_path):
    ensure("clover_step", "b200")
    dumps = {}
    for tag, env in (("default", {}), ("tuned", AUTOTUNE)):
        dumps[tag] = str(tmp_path / ("%s.dump" % tag))
        r = subprocess.run([sys.executable, "-m", "apps.clover_run", "--flavour", "b200",
                            "--cells", "120", "--steps", "12", "--dump", dumps[tag]], cwd=ROOT,
                           env=dict(os.environ, **env), capture_output=True, text=True,
                           timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
    same(dumps["tuned"], dumps["default"])
