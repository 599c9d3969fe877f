"""Stand-in for ``refidxdb`` (material database), TEST ONLY. Only the reference's
config loader uses it (yasfpy/config.py:18); nothing on the coupling path does."""
