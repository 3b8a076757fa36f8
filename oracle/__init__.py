"""CPU oracle of the SGM stereo path -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and the cpu_baseline / reference arms of
bench.py. The product library never loads it.
"""
