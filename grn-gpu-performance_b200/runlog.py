"""Run persistence for the island search: an SQLite file with the tables and
columns the reference's search writes (Individual::submit,
Src/Search/individual.cpp:117-127; Generation::submit,
Src/Search/generation.cpp:96-113; the GenerationIndividual link table,
generation.cpp:85-93), models in the reference's text form
(grn_model_format), and a resume that loads a recorded generation back into
a search (grn_evolution_set_individual).

The reference's database schema itself is not part of its sources; the table
and column names here are the ones its submit() calls use.
"""
import sqlite3

import numpy as np

import grn_b200 as grn

_SCHEMA = """
CREATE TABLE IF NOT EXISTS Individual (
  Id INTEGER PRIMARY KEY, Model TEXT NOT NULL, Complexity INTEGER, Error REAL,
  SimTime REAL, Parent1 INTEGER, Parent2 INTEGER);
CREATE TABLE IF NOT EXISTS Generation (
  Id INTEGER PRIMARY KEY, Deme INTEGER NOT NULL, Ind INTEGER NOT NULL, Time REAL,
  MinError REAL, MeanError REAL, MaxError REAL,
  MinComp INTEGER, MeanComp REAL, MaxComp INTEGER, BestComp INTEGER);
CREATE TABLE IF NOT EXISTS GenerationIndividual (
  Generation INTEGER NOT NULL, Individual INTEGER NOT NULL, Position INTEGER NOT NULL);
CREATE TABLE IF NOT EXISTS SearchCheckpoint (
  Ind INTEGER PRIMARY KEY, State BLOB NOT NULL, Surrogate BLOB);
"""


class RunLog:
    """Records generations of a grn_b200.Evolution; `precision` is the
    number of significant digits of the model strings (6: what the
    reference writes; 17: exact)."""

    def __init__(self, path, precision=6):
        self.db = sqlite3.connect(path)
        self.db.executescript(_SCHEMA)
        self.precision = precision

    def close(self):
        self.db.commit()
        self.db.close()

    def record_generation(self, evo, n_demes, deme_size, generation, time_s=0.0,
                          checkpoint=False, surrogate=None):
        """One Generation row per deme (its error and complexity statistics,
        Generation::submit's values) plus its individuals; with `checkpoint`
        also the search's exact state (grn_evolution_checkpoint, a table the
        reference does not have), from which resume continues the run as it
        would have gone on; `surrogate` (the search's screen, if any) is
        checkpointed with it."""
        cur = self.db.cursor()
        for d in range(n_demes):
            inds = [evo.individual(d, i) for i in range(deme_size)]
            errs = np.array([e for _, _, e, _ in inds])
            comps = np.array([c for _, _, _, c in inds])
            best = int(np.lexsort((comps, errs))[0])  # min error, then min complexity
            cur.execute(
                "INSERT INTO Generation (Deme, Ind, Time, MinError, MeanError, MaxError, MinComp,"
                " MeanComp, MaxComp, BestComp) VALUES (?,?,?,?,?,?,?,?,?,?)",
                (d, generation, time_s, float(errs.min()), float(errs.mean()),
                 float(errs.max()), int(comps.min()), float(comps.mean()), int(comps.max()),
                 int(comps[best])))
            gen_id = cur.lastrowid
            for pos, (prods, links, err, comp) in enumerate(inds):
                cur.execute(
                    "INSERT INTO Individual (Model, Complexity, Error, SimTime) VALUES (?,?,?,?)",
                    (grn.format_model(prods, links, self.precision), int(comp), float(err), 0.0))
                cur.execute("INSERT INTO GenerationIndividual VALUES (?,?,?)",
                            (gen_id, cur.lastrowid, pos))
        if checkpoint:
            sur = sqlite3.Binary(surrogate.checkpoint()) if surrogate is not None else None
            cur.execute("INSERT OR REPLACE INTO SearchCheckpoint VALUES (?,?,?)",
                        (generation, sqlite3.Binary(evo.checkpoint()), sur))
        self.db.commit()

    def generations(self):
        """Recorded generation numbers, ascending."""
        rows = self.db.execute("SELECT DISTINCT Ind FROM Generation ORDER BY Ind").fetchall()
        return [r[0] for r in rows]

    def load_population(self, generation):
        """{deme: [(products, links, error), ...]} of a recorded generation."""
        rows = self.db.execute(
            "SELECT g.Deme, gi.Position, i.Model, i.Error FROM Generation g"
            " JOIN GenerationIndividual gi ON gi.Generation = g.Id"
            " JOIN Individual i ON i.Id = gi.Individual WHERE g.Ind = ?"
            " ORDER BY g.Deme, gi.Position", (generation,)).fetchall()
        pop = {}
        for deme, _, text, err in rows:
            prods, links = grn.parse_model(text)
            pop.setdefault(deme, []).append((prods, links, err))
        return pop

    def resume(self, evo, generation, surrogate=None):
        """Loads a recorded generation into `evo` (same deme count and size).
        Where the generation was recorded with its checkpoint, the search
        continues exactly as the recorded run did (given a deterministic
        evaluator).  Otherwise only the populations and their errors load,
        and the search's random state starts afresh, so the continuation
        differs from the original run's.  `surrogate` receives the recorded
        surrogate state, where there is one."""
        row = self.db.execute("SELECT State, Surrogate FROM SearchCheckpoint WHERE Ind = ?",
                              (generation,)).fetchone()
        if row is not None:
            evo.restore(bytes(row[0]))
            if surrogate is not None and row[1] is not None:
                surrogate.restore(bytes(row[1]))
            return
        for deme, inds in self.load_population(generation).items():
            for i, (prods, links, err) in enumerate(inds):
                evo.set_individual(deme, i, prods, links, err)
        evo.set_generation(generation)
