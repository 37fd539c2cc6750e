"""Add the missing ``return 0;`` to ParVec::initialize_data in the oracle's
build copy of include/parvec.hpp (reference lines 63-66).  Falling off the
end of that non-void function is undefined behaviour that GCC 13 -O3 turns
into a crash; the fix changes no arithmetic.  Test infrastructure only."""
import re
import sys

path = sys.argv[1]
src = open(path).read()
pat = re.compile(r"(int initialize_data\(\) \{\s*_kbytes_received = 0;\s*_kbytes_sent = 0;)(\s*\})")
new, n = pat.subn(r"\1 return 0;\2", src)
if n != 1:
    sys.exit("patch_parvec: pattern not found exactly once (found %d)" % n)
open(path, "w").write(new)
