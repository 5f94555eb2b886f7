"""TEST INFRASTRUCTURE ONLY: the CPU oracle (a C++ restatement of vexq's
exec path) and the reference's own filter kernel built from its sources.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it."""
