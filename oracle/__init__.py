"""ORACLE / TEST INFRASTRUCTURE ONLY.

The CPU checker for the B200 pressure projection: ``oracle.cpu`` wraps the plain-C restatement of the NEREUS
pressure path (``pressure_oracle.c``); ``oracle.refcase`` drives the reference's own code, compiled from its sources
by ``oracle/Makefile`` into ``oracle/_ref/``. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg import this package, and only to check or to time a baseline; the product path never does.
"""
