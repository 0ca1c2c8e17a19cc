"""Test oracle package (TEST INFRASTRUCTURE ONLY): a CPU restatement of the
reference's AMG path, used by tests/, smoke() and bench.py's CPU legs."""
