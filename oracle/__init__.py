"""CPU oracle for the Huffman-with-gap-arrays path.

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use it as the checker.  The product package never imports it.
"""
