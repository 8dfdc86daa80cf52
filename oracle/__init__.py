"""Test infrastructure: the CPU checkers of the contact path (see native.py)."""
