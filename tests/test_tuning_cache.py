"""The autotuner's cache file (host logic, no GPU): it round-trips, an
unreadable file reads as empty, and processes writing it at the same time
always leave a whole JSON file behind."""

import json
import multiprocessing as mp

from qj.core import read_tuning_cache, write_tuning_cache


def test_roundtrip_and_missing(tmp_path):
    path = tmp_path / "sub" / "tuning.json"
    assert read_tuning_cache(str(path)) == {}
    write_tuning_cache(str(path), {"B200|256|256|256|1|4096|1": [0, 1, 2]})
    assert read_tuning_cache(str(path)) == {"B200|256|256|256|1|4096|1": [0, 1, 2]}
    assert [p.name for p in path.parent.iterdir()] == ["tuning.json"]  # no temporary left


def test_cut_short_file_reads_as_empty(tmp_path):
    path = tmp_path / "tuning.json"
    path.write_text('{"B200|64|64|64|1|0|1": [0, ')
    assert read_tuning_cache(str(path)) == {}
    path.write_text("[1, 2]")
    assert read_tuning_cache(str(path)) == {}


def _writer(path, who, n):
    for i in range(n):
        cache = read_tuning_cache(path)
        cache[f"{who}|{i}"] = list(range(10))
        write_tuning_cache(path, cache)


def test_concurrent_writers_leave_whole_json(tmp_path):
    path = str(tmp_path / "tuning.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, w, 40)) for w in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    with open(path) as f:
        cache = json.load(f)  # a whole file, whichever writer was last
    assert any(k.endswith("|39") for k in cache)
