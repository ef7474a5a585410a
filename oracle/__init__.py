"""Test infrastructure: the CPU oracle (a restatement of the reference's CPU
codecs) and the loader for the reference's own CPU build (oracle/_ref).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this package; the product library never imports it."""
