#!/bin/bash
# Compile the reference's own hot-path C sources (read in place from the
# reference tree, never copied) plus oracle/ref_harness.c into
# oracle/_ref/libpinyref.so.  Test infrastructure only; needs the reference
# tree, so it runs in the build container and the resulting .so travels.
set -e
REF=${SDFT_REFERENCE_DIR:-}
[ -n "$REF" ] || { echo "SDFT_REFERENCE_DIR is not set: the reference-compiled oracle is not built"; exit 0; }
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
[ -d "$REF/stodft" ] || { echo "reference tree not found at $REF"; exit 0; }
mkdir -p "$OUT/obj"
INC="-I$HERE/ref_stubs -I$REF/include/pentium_nopar -include $HERE/ref_stubs/sdft_ref_protos.h"
CFLAGS="-O2 -fPIC -w -ffp-contract=off"
SRCS="stodft/filter.c stodft/normh.c stodft/calc-chempot-chebyshev.c stodft/coeff.c
      stodft/reduced-energy/energy-wrapper-scf.c stodft/reduced-energy/cp-energy-eext-stodft.c
      stodft/reduced-energy/cp-energy-ee-rho-stodft.c mathlib/fft_package.c mathlib/fft_create_package.c
      mathlib/mathlib.c energy/cp/cp_energy_eext_nonloc.c energy/cp/cp_energy_eext.c
      energy/cp/cp_energy_ee_rho.c interface/cp_ewald/set_cp_ewald.c friend_lib/cmalloc.c
      stodft/density.c stodft/gen-noise.c stodft/diis.c stodft/checkpointIO.c energy/cp/xc_functionals.c
      stodft/reduced-energy/energy-wrapper-post-scf.c interface/inter_params/spline_fit.c"
OBJS=""
for f in $SRCS; do
  o="$OUT/obj/$(echo "$f" | tr '/' '_').o"
  # the harness injects noise into calcChebyMoments through genNoiseOrbitalReal,
  # so the reference's own generator is compiled under another name
  EXTRA=""
  [ "$f" = "stodft/gen-noise.c" ] && EXTRA="-DgenNoiseOrbitalReal=ref_genNoiseOrbitalReal"
  # checkpointIO.c uses the MPI datatype names without declaring them (a
  # single-rank build never reaches the MPI calls)
  [ "$f" = "stodft/checkpointIO.c" ] && EXTRA="-DMPI_DOUBLE=1 -DMPI_INT=2"
  if [ ! -f "$o" ] || [ "$REF/$f" -nt "$o" ]; then gcc -c $CFLAGS $EXTRA $INC "$REF/$f" -o "$o"; fi
  OBJS="$OBJS $o"
done
gcc -c $CFLAGS $INC "$HERE/ref_harness.c" -o "$OUT/obj/ref_harness.o"
gcc -shared -o "$OUT/libpinyref.so" $OBJS "$OUT/obj/ref_harness.o" -lm
echo "$OUT/libpinyref.so"

# The product's PINY adapter (csrc/piny/sdft_piny_adapter.c), compiled against
# the reference headers and linked in place of the reference routines it
# replaces: the same objects with those definitions made weak, the same
# harness, and lib/libsdft_b200.so.  The reference's own callers (the
# harness drives them) then run on the device path.
PKG="$(cd "$HERE/.." && pwd)/stochastic-density-functional-theory-piny_b200"
if [ -f "$PKG/lib/libsdft_b200.so" ]; then
  mkdir -p "$OUT/obj_adapter"
  WEAK=""
  for sym in filterChebyPolyHerm filterNewtonPolyHerm normHCheby normHNewtonHerm calcChebyMoments \
             calcCoefForceWrapSCF rhoCalcRealStoHybrid; do WEAK="$WEAK --weaken-symbol=$sym"; done
  AOBJS=""
  for o in $OBJS; do
    w="$OUT/obj_adapter/$(basename "$o")"
    objcopy $WEAK "$o" "$w"
    AOBJS="$AOBJS $w"
  done
  # the harness supplies genNoiseOrbitalReal here (it injects chi into calcChebyMoments);
  # the adapter's noise is reached through sdft_piny_noise
  gcc -c $CFLAGS -DSDFT_PINY_ADAPTER -DSDFT_PINY_ADAPTER_NO_NOISE $INC -I"$REF/stodft" -I"$HERE/../include" \
      "$PKG/csrc/piny/sdft_piny_adapter.c" -o "$OUT/obj_adapter/sdft_piny_adapter.o"
  gcc -shared -o "$OUT/libpinyref_adapter.so" $AOBJS "$OUT/obj/ref_harness.o" \
      "$OUT/obj_adapter/sdft_piny_adapter.o" -L"$PKG/lib" -lsdft_b200 \
      -Wl,-rpath,'$ORIGIN/../../stochastic-density-functional-theory-piny_b200/lib' -lm
  echo "$OUT/libpinyref_adapter.so"
  # the production form (with genNoiseOrbitalReal) compiles against the same headers
  gcc -c $CFLAGS -DSDFT_PINY_ADAPTER $INC -I"$REF/stodft" -I"$HERE/../include" \
      "$PKG/csrc/piny/sdft_piny_adapter.c" -o "$OUT/obj_adapter/sdft_piny_adapter_full.o"
fi
