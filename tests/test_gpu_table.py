"""Table mode end to end on the GPU: the CLI with -tb runs every job of the
table, writes the same .out files as single-job runs of the same command
lines, retries a failing job with the ".retry" output suffix and reports
both in the log's JOB and Worker tables (src/mpidp.cpp:880-914 format)."""
import subprocess

import pytest

pytestmark = pytest.mark.gpu


def test_table_jobs_match_single_runs(built, gpu, pairs, tmp_path):
    from megadock_b200 import _native
    (r0, l0), (r1, l1) = pairs["small"], pairs["c0"]
    tb = tmp_path / "jobs.table"
    outs = [tmp_path / "a.out", tmp_path / "b.out", tmp_path / "c.out"]
    tb.write_text("TITLE=three jobs\nPARAM=-R $1 -L $2 -o $3 -F 96\n"
                  f"{r0}\t{l0}\t{outs[0]}\n{r1}\t{l1}\t{outs[1]}\n{tmp_path}/missing_r.pdb\t{l0}\t{outs[2]}\n")
    log = tmp_path / "master.log"
    res = subprocess.run([str(_native.CLI_PATH), "-tb", str(tb), "-ot", "3", "-rt", "1", "-lg", str(log),
                          "-r", "360", "-N", "100"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 1, res.stderr          # one job cannot succeed
    assert "2 of 3 jobs" in res.stdout
    text = log.read_text()
    assert "TITLE=three jobs" in text and "PARAM=-R $1 -L $2 -o $3 -F 96" in text
    assert "Other options : -r 360 -N 100" in text
    jobs = text.split("JOB table :\n")[1].split("\n\n")[0].splitlines()
    assert jobs[0] == "00001\t EXEC=1 (WID=1 END=1 RET=0 FILE=1)"
    assert jobs[1] == "00002\t EXEC=1 (WID=1 END=1 RET=0 FILE=1)"
    assert jobs[2].startswith("00003\t EXEC=2 (WID=1 END=1 RET=") and jobs[2].endswith("FILE=-1)")
    assert jobs[2].count("WID=1") == 2
    worker = text.split("Worker table :\n")[1].splitlines()
    assert worker[0] == "no.\t#exec\tdetail"
    assert worker[1].startswith("1\t4\t00001\t\t1\t00002\t\t1\t00003\t\t1\t00003\t\t1")
    for (rp, lp), out in zip([(r0, l0), (r1, l1)], outs[:2]):
        single = tmp_path / ("single_" + out.name)
        r = subprocess.run([str(_native.CLI_PATH), "-R", rp, "-L", lp, "-o", str(single), "-F", "96", "-r", "360",
                            "-N", "100"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        assert out.read_text() == single.read_text()
