"""Test infrastructure only: the CPU oracle (C++ restatement of the reference
megakernel) and its build recipe.  Imported by tests/, __graft_entry__.smoke()
and bench.py's CPU baseline; never by the mutracer_b200 package."""
