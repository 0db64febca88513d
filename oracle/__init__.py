"""Test-only CPU oracle of the slab Foldy-Lax path (see slab_oracle.py).

Never imported by the shipped package.
"""
