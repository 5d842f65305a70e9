#!/bin/bash
# ORACLE recipe — test infrastructure only.
#
# Compiles the reference's kriging sources, where they lie under the read-only
# reference checkout, into oracle/_ref/libhpgl_ref.so (git-ignored; it is
# copied along with the working tree to the machine that runs the GPU tests).
# Nothing from the reference is copied into this repository: the shim headers
# in oracle/ref_shim/ stand in for boost (boost::mt11213b restated from its
# published parameters) and the CLAPACK headers, oracle/lapack_restated.c
# supplies dpotrf_/dpotrs_, and oracle/gen_primes.py writes the prime table
# the sequential simulation's path generator includes (primes.txt, missing
# from the checkout: every prime in increasing order past 10^7).
#
# Flags: -O2 -fopenmp as the reference's release build (SConstruct:23-24),
# with -ffp-contract=off instead of -march=native so that no a*b+c is fused.
set -euo pipefail
REF=${HPGL_REFERENCE_SRC:-/root/reference/src}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
if [ ! -d "$REF/geo_bsd/hpgl" ]; then
    echo "reference sources not found at $REF; oracle/_ref not built" >&2
    exit 3
fi
mkdir -p "$OUT/obj"
mkdir -p "$OUT/gen"
[ -s "$OUT/gen/primes.txt" ] || python3 "$HERE/gen_primes.py" "$OUT/gen/primes.txt"
CXXFLAGS="-std=gnu++11 -O2 -fopenmp -ffp-contract=off -fPIC -w -DNDEBUG -I$OUT/gen -I$HERE/ref_shim -I$REF/tnt_126 -I$REF/geo_bsd/hpgl"
TUS="api.cpp api_helpers.cpp ordinary_kriging.cpp simple_kriging.cpp lvm_kriging.cpp indicator_kriging.cpp
median_ik.cpp clusterizer.cpp covariance_field.cpp covariance_param.cpp neighbourhood_param.cpp ok_params.cpp
sk_params_t.cpp ik_params.cpp calc_mean.cpp cdf_utils.cpp mean_provider.cpp output.cpp pretty_printer.cpp
progress_reporter.cpp kriging_stats.cpp hpgl_exception.cpp sugarbox_grid.cpp set_thread_num.cpp
property_writer.cpp read_inc_file.cpp simple_cokriging_markI.cpp sgs_params.cpp bs_assert.cpp logging.cpp
gauss_solver.cpp load_property_from_file.cpp path_random_generator.cpp bs_random_generator.cpp
sequential_gaussian_simulation.cpp sequential_indicator_simulation.cpp sample.cpp random_node_enumerator.cpp"
pids=()
for f in $TUS; do
    g++ $CXXFLAGS -c "$REF/geo_bsd/hpgl/$f" -o "$OUT/obj/${f%.cpp}.o" &
    pids+=($!)
done
g++ $CXXFLAGS -c "$HERE/ref_dump.cpp" -o "$OUT/obj/ref_dump.o" & pids+=($!)
gcc -O2 -ffp-contract=off -fPIC -c "$HERE/lapack_restated.c" -o "$OUT/obj/lapack_restated.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
rm -f "$OUT/obj/ref_stubs.o"
g++ -shared -fopenmp -o "$OUT/libhpgl_ref.so" "$OUT"/obj/*.o
echo "built $OUT/libhpgl_ref.so"

# The experimental-variogram library (_cvariogram: variograms.cpp,
# ellipsoid.cpp, stack_layers.cpp) as the reference builds it
# (_cvariogram/SConstruct: no optimisation flags there; -O2 -ffp-contract=off
# here as for the kriging sources), plus oracle/ref_cvar_shim.cpp.
CV=$REF/geo_bsd/_cvariogram
mkdir -p "$OUT/cvobj"
CVFLAGS="-std=gnu++11 -O2 -ffp-contract=off -fPIC -w -DNDEBUG -I$CV"
for f in variograms.cpp ellipsoid.cpp stack_layers.cpp; do
    g++ $CVFLAGS -c "$CV/$f" -o "$OUT/cvobj/${f%.cpp}.o"
done
g++ $CVFLAGS -c "$HERE/ref_cvar_shim.cpp" -o "$OUT/cvobj/ref_cvar_shim.o"
g++ -shared -o "$OUT/libcvariogram_ref.so" "$OUT"/cvobj/*.o
echo "built $OUT/libcvariogram_ref.so"
