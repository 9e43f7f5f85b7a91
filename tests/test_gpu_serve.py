"""Continuous batching: jobs that arrive while others run are admitted between
chunks, run together with them, and finish with exactly the result they give
alone (mixed form: bit for bit)."""
import numpy as np
import pytest

from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine
from mjolnir_b200.serve import Job, Server, poisson_workload

pytestmark = pytest.mark.gpu


def alone(desc, nsteps):
    e = Engine("mixed")
    sid = e.add_system(desc)
    e.commit()
    e.step(nsteps)
    p, v, _ = e.state(sid)
    e.close()
    return p, v


def test_jobs_same_alone_and_in_the_mix():
    specs = [
        (S.polymer_melt(nchains=3, nbeads=60, radius=45.0, seed=71, temperature=290.0), 230),
        (S.polymer_melt(nchains=2, nbeads=80, radius=40.0, seed=72, temperature=350.0,
                        ionic_strength=0.2), 410),
        (S.bead_fluid(n=1500, density=0.003, seed=73, dt=0.3), 170),
        (S.lj_fluid(n=512, seed=74), 300),
    ]
    srv = Server(precision="mixed", chunk=100)
    jobs = [Job(job_id=k, nsteps=n, arrival=0.0, desc=d.copy()) for k, (d, n) in enumerate(specs)]
    srv.submit(jobs[0])
    srv.submit(jobs[1])
    for _ in range(2):          # the first two run alone for a while
        srv.step_once()
    srv.submit(jobs[2])
    srv.step_once()
    srv.submit(jobs[3])
    srv.run_until_idle(timeout=120)
    assert len(srv.finished) == 4
    for j, (d, n) in zip(jobs, specs):
        assert j.done == n
        p, v = alone(d, n)
        assert np.array_equal(j.pos, p), j.job_id
        assert np.array_equal(j.vel, v), j.job_id
    st = srv.stats(srv.now())
    assert st["completed"] == 4 and st["latency_p50_s"] is not None
    srv.close()


def test_admission_respects_memory_budget():
    srv = Server(precision="mixed", chunk=50)
    srv.budget = 1.0                     # room for one job at a time
    descs = [S.polymer_melt(nchains=2, nbeads=40, radius=35.0, seed=80 + k) for k in range(3)]
    for k, d in enumerate(descs):
        srv.submit(Job(job_id=k, nsteps=60, arrival=0.0, desc=d))
    srv.step_once()
    assert len(srv.running) == 1 and len(srv.queue) == 2
    srv.run_until_idle(timeout=120)
    assert len(srv.finished) == 3
    srv.close()


def test_poisson_workload_shape():
    jobs = poisson_workload(rate=200.0, duration=1.0, seed=3)
    assert 120 < len(jobs) < 300
    assert all(1000 <= j.nsteps <= 100000 for j in jobs)
    d = jobs[0].build()
    assert 150 <= d.n <= 60000
