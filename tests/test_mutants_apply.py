"""The mutation check's mutants still apply to the sources (each text occurs exactly once), so
tests/mutation_check.py stays runnable as the code changes."""
import mutation_check


def test_every_mutant_applies():
    assert mutation_check.stale() == []
    assert len({m[0] for m in mutation_check.MUTANTS}) == len(mutation_check.MUTANTS)
