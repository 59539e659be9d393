"""The training log <name>.log (logger.cpp:31-74): a header line of the
logged names, then one line per applied update with energy per spin, its
standard deviation per spin and the acceptance rate (the values of
stochastic_reconfiguration.cpp:86-91 and metropolis_sampler.cpp:275-277),
at 16 significant digits."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def session(**kw):
    rng = np.random.default_rng(3)
    om = O.Model.kitaev(3)
    mach = O.Machine(om, "basic", 1, symm=0.5).init_random(rng, 0.05)
    base = dict(rbm_type=0, alpha=1, n_chains=16, samples_per_chain=8, warmup=4, seed=5, precision=1)
    base.update(kw)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(3), rbmnqs.default_config(**base))
    s.set_weights(mach.params())
    return s


def read_log(path):
    lines = open(path).read().splitlines()
    return lines


def test_log_lines_follow_the_epochs(tmp_path):
    s = session()
    name = str(tmp_path / "kitaev3")
    s.log_open(name)
    stats = []
    for _ in range(3):
        st, sr = s.epoch()
        assert sr["status"] == 0
        stats.append(st)
    s.log_close()
    lines = read_log(name + ".log")
    assert lines[0] == "# Energy, Energy Stddev, AccetpanceRate"
    assert len(lines) == 4
    n = 18
    for line, st in zip(lines[1:], stats):
        vals = [float(v) for v in line.split(", ")]
        assert vals == [float("%.16g" % (st["energy"].real / n)), float("%.16g" % (st["stddev"] / n)),
                        float("%.16g" % st["acceptance"])]
    # stepwise sample + optimize writes the same kind of line
    s.log_open(name)  # exists, no force: append, with a new header
    s.sample()
    s.optimize()
    s.log_close()
    lines = read_log(name + ".log")
    assert len(lines) == 6 and lines[4].startswith("# Energy")
    # force truncates
    s.log_open(name, force=True)
    s.epoch()
    s.log_close()
    assert len(read_log(name + ".log")) == 2


def test_sgd_and_full_sampler_headers(tmp_path):
    s = session(optimizer_type=1)
    s.log_open(str(tmp_path / "sgd"))
    s.epoch()
    s.log_close()
    assert read_log(str(tmp_path / "sgd.log"))[0] == "# Energy, EnergyStddev, AccetpanceRate"
    f = session(sampler_type=1)
    f.log_open(str(tmp_path / "full"))
    f.epoch()
    f.log_close()
    lines = read_log(str(tmp_path / "full.log"))
    assert lines[0] == "# Energy, Energy Stddev" and len(lines[1].split(", ")) == 2


def test_rejected_step_writes_no_line(tmp_path):
    """A step rejected by the max|dw| > 30 guard leaves the log as it was
    (main.cpp:600-616 stops before logger::newline)."""
    s = session(optimizer_type=1, sgd_real_factor=1e-9)
    s.log_open(str(tmp_path / "massive"))
    st, sr = s.epoch()
    assert sr["status"] == rbmnqs.ERR_MASSIVE_STEP
    s.log_close()
    assert read_log(str(tmp_path / "massive.log")) == []
