#!/bin/bash
# Builds the reference's own DGSEM sources, unmodified, from where they lie
# under the reference checkout (REF, default /root/reference) against the MFEM
# stand-in in mfem_standin/, into oracle/_ref/libref_<variant>.so.  One library
# per compile-time physics switch set of the reference (PARABOLIC,
# SUBCELL_FV_BLENDING; SUTHERLAND off), as its CMake build would configure.
# Test infrastructure only: the outputs are the parity pin of the CPU oracle.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/../_ref"
SRC="$REF/src"
if [ ! -d "$SRC" ]; then
  echo "reference sources not found at $SRC; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX="${CXX_REF:-g++}"
INC="-I$HERE/mfem_standin -I$HERE/.. -I$SRC/BasicOperations -I$SRC/RiemannSolvers -I$SRC/Fluxes \
 -I$SRC/Integrators/DGSEMIntegrator -I$SRC/Integrators/Lifting -I$SRC/Integrators/Lifting/LiftingBR1 \
 -I$SRC/Integrators/BoundaryConditions -I$SRC/Indicators -I$SRC/ModalBasis -I$SRC/Physics"
FILES="$SRC/BasicOperations/BasicOperations.cpp $SRC/RiemannSolvers/ChandrashekarFlux.cpp \
 $SRC/Fluxes/NavierStokesFlux.cpp $SRC/Integrators/DGSEMIntegrator/DGSEMIntegrator.cpp \
 $SRC/Integrators/Lifting/LiftingScheme.cpp $SRC/Integrators/Lifting/LiftingBR1/LiftingBR1.cpp \
 $SRC/Indicators/Indicator.cpp $SRC/Indicators/PerssonPeraireIndicator.cpp $SRC/ModalBasis/ModalBasis.cpp \
 $SRC/Integrators/BoundaryConditions/BdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SpecifiedStateBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SupersonicOutflowBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SlipWallBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SymmetryBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SubsonicOutflowPBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/RiemannInvariantBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SubsonicInflowRVBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SubsonicInflowPtTtAngBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/NoSlipAdiabWallBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/NoSlipIsothWallBdrFaceIntegrator.cpp \
 $HERE/ref_driver.cpp"
# -O2 -DNDEBUG as the reference's Release configuration (configure.sh)
FLAGS="-O2 -DNDEBUG -std=c++17 -fPIC -shared -w"
build() {
  local name="$1"; shift
  $CXX $FLAGS "$@" $INC $FILES -o "$OUT/libref_$name.so"
}
# the six variants compile in parallel; any failure fails the script
pids=()
build euler & pids+=($!)
build euler_blend -DSUBCELL_FV_BLENDING & pids+=($!)
build ns -DPARABOLIC & pids+=($!)
build ns_blend -DPARABOLIC -DSUBCELL_FV_BLENDING & pids+=($!)
build euler_axi -DAXISYMMETRIC & pids+=($!)
build euler_blend_axi -DSUBCELL_FV_BLENDING -DAXISYMMETRIC & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
echo "built $(ls "$OUT"/libref_*.so | wc -l) reference libraries in $OUT"
