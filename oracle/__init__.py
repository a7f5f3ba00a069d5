"""CPU oracle of the likelihood path (test infrastructure; see binding.py)."""
