"""CPU oracle of GITM's vertical advance -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py import
this package; the product library never does.
"""
