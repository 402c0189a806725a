"""Host-side helpers of bench.py: the CPU-baseline sample sizing, the
whole-job rate, the algorithmic byte model of the roofline and the serving
mix's handling of jobs that do not finish."""
import os
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_scaled_sample_targets_seconds_and_caps_at_the_workload():
    wl = bench.WORKLOADS["ns"]
    # 200k reads with 120 k-mers each at 80 M k-mers/s -> 10 s is 6.67 M reads
    n = bench.scaled_sample(wl, 200_000, 24_000_000, 80e6, 10.0)
    assert n == pytest.approx(80e6 * 10 / 120, rel=1e-6)
    assert bench.scaled_sample(wl, 200_000, 24_000_000, 1e12, 10.0) == 20_000_000  # all reads of the workload
    assert bench.scaled_sample(wl, 200_000, 24_000_000, 1.0, 10.0) == 200_000     # never below the calibration
    assert bench.scaled_sample(bench.WORKLOADS["config1"], 100, 12_000, 1e12, 10.0) == 20_000


def test_whole_job_rate_counts_every_rank():
    assert bench.whole_job_rate(100, 4, 2, 1000.0) == pytest.approx(800.0)


def test_byte_model_at_ns():
    m = bench.algorithmic_bytes(3.0e9, 2e7, 2.28e8, 2.4e9, 4.36e8, 31)
    assert m["w"] == 8 and m["P"] == 8
    assert m["sort"] == pytest.approx(8 * 2.4e9 * (1 + 2 * 8))
    assert m["count"] == pytest.approx(8 * 2.4e9 + 12 * 4.36e8)
    assert m["total"] == pytest.approx(m["partition"] + m["expand"] + m["sort"] + m["count"])
    assert bench.algorithmic_bytes(1, 1, 1, 1, 1, 63)["w"] == 16


class _Info:
    def __init__(self, state, n_bases=0, submit_s=0.0, end_s=0.0):
        self.state, self.status, self.n_bases, self.n_kmers = state, 0 if state == 2 else 3, n_bases, n_bases
        self.submit_s, self.end_s = submit_s, end_s


class _FakeServer:
    """Stands in for gkc_b200.Server: every job finishes at once except the
    ids in `never`, which stay running (a worker that does not come back)."""

    def __init__(self, device, max_running=4, never=()):
        self.jobs, self.never, self.closed, self.next = {}, set(never), False, 1

    def _add(self, n_bases):
        j = self.next
        self.next += 1
        t = time.perf_counter()
        self.jobs[j] = _Info(1 if j in self.never else 2, n_bases, t, t + 0.001)
        return j

    def submit(self, reads, offs, prm):
        return self._add(int(offs[-1]))

    def submit_synth(self, prm, g, seed, n_bases):
        return self._add(int(n_bases))

    def wait(self, j, timeout=-1.0):
        if self.jobs[j].state == 1:
            time.sleep(min(timeout, 0.01) if timeout >= 0 else 0.01)
        return self.jobs[j]

    def release(self, j):
        assert self.jobs[j].state != 1
        del self.jobs[j]

    def close(self):
        self.closed = True


def _fake_module(never):
    import types
    import gkc_b200 as G
    made = []

    def server(device, max_running=4):
        made.append(_FakeServer(device, max_running, never))
        return made[-1]
    return types.SimpleNamespace(Server=server, params=G.params, lib=G.lib), made


def test_serving_mix_reports_a_job_that_never_finishes():
    """A job whose worker never returns is reported as unfinished after the
    grace period (the mix does not wait for it), and the server is left
    open for the caller to end the process."""
    fake, made = _fake_module(never={7})
    out = bench.serve_mix(fake, 0, 12, (0.8,), 5, calib_jobs=4, host_pool_bases=300_000, grace_s=0.2)
    l80 = out["loads"]["0.80"]
    assert out["stuck"] is True and not made[0].closed
    assert l80["unfinished_count"] == 1 and l80["unfinished"][0]["job"] == 7
    assert l80["unfinished"][0]["state"] == "running"
    assert l80["failed"] == 0 and l80["jobs"] == 12


def test_serving_mix_closes_the_server_when_every_job_ends():
    fake, made = _fake_module(never=())
    out = bench.serve_mix(fake, 0, 12, (0.8,), 5, calib_jobs=4, host_pool_bases=300_000, grace_s=0.2)
    assert out["stuck"] is False and made[0].closed
    assert out["loads"]["0.80"]["unfinished_count"] == 0


def test_serving_child_results_and_failures(monkeypatch):
    """The default run's serving leg: the child's serving object, its exit
    code when it left jobs unfinished, and an error (never a hang) when it
    times out or prints no line."""
    import subprocess
    import types
    args = types.SimpleNamespace(serve_jobs=None, seed=5, serve_timeout=1.0)
    line = '{"metric": "m", "serving": {"loads": {}, "stuck": true}}'

    def done(rc, out):
        return lambda cmd, **kw: subprocess.CompletedProcess(cmd, rc, out, "tail")
    monkeypatch.setattr(bench.subprocess, "run", done(3, "noise\n" + line + "\n"))
    res = bench.serve_child(args)
    assert res["stuck"] is True and res["exit_code"] == 3
    monkeypatch.setattr(bench.subprocess, "run", done(0, line))
    assert "exit_code" not in bench.serve_child(args)
    monkeypatch.setattr(bench.subprocess, "run", done(1, "no json here"))
    assert "without a result" in bench.serve_child(args)["error"]

    def late(cmd, **kw):
        assert kw["timeout"] == 1.0 and "--serve" in cmd and "0.8" in cmd
        raise subprocess.TimeoutExpired(cmd, kw["timeout"], output="", stderr="stuck")
    monkeypatch.setattr(bench.subprocess, "run", late)
    res = bench.serve_child(args)
    assert "did not finish within 1 s" in res["error"] and res["stderr_tail"] == "stuck"
