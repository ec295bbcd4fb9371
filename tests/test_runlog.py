"""The driver's run log: records are one line each and parse back."""

import logging

from pygsquig_b200.utils.runlog import RunLog, parse_record


def test_records_parse_back(tmp_path, capsys):
    log = RunLog(tmp_path, level="DEBUG")
    log.event("progress", t=1.25, step=40, dt=2e-4, energy=0.5)
    log.event("resume", file="a b.h5", step=3)
    log.event("wall_limit", logging.WARNING, limit_s=60)
    lines = (tmp_path / "logs" / "run.log").read_text().splitlines()
    assert len(lines) == 3
    r = parse_record(lines[0])
    assert r == {"event": "progress", "t": "1.25", "step": "40", "dt": "0.0002", "energy": "0.5"}
    assert parse_record(lines[1]) == {"event": "resume", "file": "a b.h5", "step": "3"}
    assert parse_record(lines[2])["event"] == "wall_limit"
    assert " W wall_limit" in lines[2]
    out = capsys.readouterr().out
    assert "progress t=1.25" in out


def test_level_filters_console_not_file(tmp_path, capsys):
    log = RunLog(tmp_path, level="WARNING")
    log.wrote("fields", tmp_path / "f.npz", 0.5, 10)
    assert capsys.readouterr().out == ""
    assert "fields file=f.npz" in (tmp_path / "logs" / "run.log").read_text()
