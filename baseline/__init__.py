"""The reference arm of `bench.py`: the reference's own CPU path, installed under `_ref`."""
