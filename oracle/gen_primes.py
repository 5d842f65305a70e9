"""ORACLE — test infrastructure only.  Writes the prime table that the
reference's path_random_generator.cpp includes as "primes.txt" (missing from
its checkout): every prime up to LIMIT in increasing order, comma-separated.
init_rnd (path_random_generator.cpp:20-56) asserts grids of at most 10^7
nodes and needs a prime above the grid size after the last factor it
checks, so the table runs a little past 10^7; it is the only table
consistent with those asserts.

    python oracle/gen_primes.py OUT [LIMIT]"""

import sys

import numpy as np


def primes_upto(n):
    sieve = np.ones(n + 1, dtype=bool)
    sieve[:2] = False
    for p in range(2, int(n ** 0.5) + 1):
        if sieve[p]:
            sieve[p * p::p] = False
    return np.nonzero(sieve)[0]


if __name__ == "__main__":
    limit = int(sys.argv[2]) if len(sys.argv) > 2 else 10000200
    with open(sys.argv[1], "w") as f:
        f.write(",\n".join(",".join(str(int(p)) for p in chunk)
                           for chunk in np.array_split(primes_upto(limit), 4000)))
        f.write("\n")
