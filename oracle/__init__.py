"""CPU oracle of pygranite's step path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, to verify
the engine's results.  The engine in pygranite_b200/ never imports, links or calls anything
here.
"""
