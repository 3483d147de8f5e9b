"""The coarse-vector training set file: round trip of its records (digests
kept byte-exact, trailing zero bytes included), magic and version checks,
and the regeneration keys the recorded-epoch trainer groups by."""
import os

import numpy as np
import pytest


def _record(design, it, seed=9000, cells=5000, sha_tail=b"\x00"):
    sha = bytes(range(31)) + sha_tail
    return dict(design=design, seed=seed + design, cells=cells, nets=5250, iteration=it,
                alpha=0.01 + 0.01 * it, n=cells, nnz_x=7 * cells, nnz_y=7 * cells,
                fp64_iters_x=100, fp64_iters_y=101, agg_iters_x=20, agg_iters_y=21,
                loss_x=0.3, loss_y=0.25, system_sha=sha, solution_sha=sha[::-1])


def test_round_trip(tmp_path):
    from ktplace_b200.learned import CoarseDataset, DATASET_VERSION
    ds = CoarseDataset()
    for d in range(2):
        for it in range(3):
            ds.add(**_record(d, it))
    path = os.path.join(tmp_path, "set.bin")
    ds.save(path)
    raw = open(path, "rb").read()
    assert raw[:8] == b"KTGCOARS"
    assert np.frombuffer(raw[8:16], dtype="<u4").tolist() == [DATASET_VERSION, 6]
    rec = CoarseDataset.load(path)
    assert len(rec) == 6
    assert rec[4]["system_sha"].tobytes() == _record(1, 1)["system_sha"]  # trailing zero kept
    assert rec[4]["solution_sha"].tobytes() == _record(1, 1)["solution_sha"]
    assert int(rec[5]["iteration"]) == 2 and int(rec[5]["design"]) == 1


def test_bad_files(tmp_path):
    from ktplace_b200.learned import CoarseDataset, DATASET_VERSION
    p = os.path.join(tmp_path, "bad.bin")
    open(p, "wb").write(b"NOTMAGIC" + bytes(8))
    with pytest.raises(ValueError):
        CoarseDataset.load(p)
    open(p, "wb").write(b"KTGCOARS" + np.array([DATASET_VERSION + 1, 0], dtype="<u4").tobytes())
    with pytest.raises(ValueError):
        CoarseDataset.load(p)


def test_dataset_designs_groups_iterations(tmp_path, monkeypatch):
    from ktplace_b200 import train_precond
    from ktplace_b200.learned import CoarseDataset
    ds = CoarseDataset()
    for it in (0, 2, 1):
        ds.add(**_record(0, it, cells=5000))
    ds.add(**_record(3, 4, cells=7000))
    path = os.path.join(tmp_path, "set.bin")
    ds.save(path)
    made = []
    monkeypatch.setattr(train_precond, "coarse_design",
                        lambda k, cells, s: made.append((k, cells, s)) or ("nl", k))
    got = list(train_precond.dataset_designs(CoarseDataset.load(path)))
    assert made == [(0, 5000, 9000), (3, 7000, 9003)]
    assert [(k, its) for k, _, its in got] == [(0, [0, 1, 2]), (3, [4])]
