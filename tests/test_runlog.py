"""Run persistence (runlog.py): generations recorded in the reference's
table layout with models in its text form, read back and resumed."""
import numpy as np

import grn_b200 as grn
import runlog
from test_evolution import EVO, SIM, OracleCalculator


def test_record_reload_resume(built_libs, tmp_path):
    calc = OracleCalculator(SIM)
    evo = grn.Evolution(dict(EVO, seed=21), 2, calculator=calc)
    log = runlog.RunLog(str(tmp_path / "run.db"), precision=17)
    for _ in range(3):
        st = evo.step()
        log.record_generation(evo, EVO["n_demes"], EVO["deme_size"], st["generation"])
    assert log.generations() == [0, 1, 2]
    rows = log.db.execute("SELECT COUNT(*) FROM Individual").fetchone()[0]
    assert rows == 3 * EVO["n_demes"] * EVO["deme_size"]
    g2 = log.db.execute("SELECT Deme, MinError, BestComp FROM Generation WHERE Ind = 2"
                        " ORDER BY Deme").fetchall()
    pop = log.load_population(2)
    for deme, min_err, best_comp in g2:
        live = [evo.individual(deme, i) for i in range(EVO["deme_size"])]
        assert min_err == min(e for _, _, e, _ in live)
        for (p1, l1, e1), (p2, l2, e2, _) in zip(pop[deme], live):
            np.testing.assert_array_equal(p1, p2)  # 17 digits: exact
            np.testing.assert_array_equal(l1, l2)
            assert e1 == e2
    # resume into a fresh search: same populations, then it keeps evolving
    evo2 = grn.Evolution(dict(EVO, seed=99), 2, calculator=OracleCalculator(SIM))
    log.resume(evo2, 2)
    for d in range(EVO["n_demes"]):
        for i in range(EVO["deme_size"]):
            a, b = evo.individual(d, i), evo2.individual(d, i)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    st = evo2.step()
    assert st["generation"] == 3 and st["best_error"] <= min(r[1] for r in g2)
    log.close()
    evo.close()
    evo2.close()


def test_resume_rejects_empty_population(built_libs):
    evo = grn.Evolution(dict(EVO, seed=1), 2, calculator=OracleCalculator(SIM))
    try:
        evo.set_generation(4)
        raise AssertionError("expected an error")
    except grn.GrnError as e:
        assert "MODEL" in str(e)
    evo.close()


def test_resume_from_a_recorded_checkpoint_is_exact(built_libs, tmp_path):
    """record_generation(checkpoint=True) stores the search's exact state;
    resume then continues as the recorded run did."""
    evo = grn.Evolution(dict(EVO, seed=23), 2, calculator=OracleCalculator(SIM))
    log = runlog.RunLog(str(tmp_path / "run.db"))
    for _ in range(3):
        st = evo.step()
        log.record_generation(evo, EVO["n_demes"], EVO["deme_size"], st["generation"],
                              checkpoint=(st["generation"] == 1))
    tail = [evo.step() for _ in range(2)]  # generations 3 and 4
    evo2 = grn.Evolution(dict(EVO, seed=5), 2, calculator=OracleCalculator(SIM))
    log.resume(evo2, 1)
    tail2 = [evo2.step() for _ in range(3)][1:]  # generations 2, 3, 4
    assert [s["generation"] for s in tail2] == [s["generation"] for s in tail] == [3, 4]
    assert [s["mean_error"] for s in tail2] == [s["mean_error"] for s in tail]
    for d in range(EVO["n_demes"]):
        for i in range(EVO["deme_size"]):
            a, b = evo.individual(d, i), evo2.individual(d, i)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    log.close()
    evo.close()
    evo2.close()

