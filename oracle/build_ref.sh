#!/bin/sh
# Builds the reference's own hot-path sources, unmodified and in place, against
# the stand-in MFEM header in oracle/ref_shim, into oracle/_ref/:
#   libref_euler.so  (-DSUBCELL_FV_BLENDING)              Euler configurations
#   libref_ns.so     (-DPARABOLIC -DSUBCELL_FV_BLENDING)  Navier-Stokes configurations
# Test infrastructure only.  Needs the reference tree (default /root/reference,
# override with PRANDTL_REFERENCE); nothing is copied out of it.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${PRANDTL_REFERENCE:-/root/reference}
SRC="$REF/src"
OUT="$HERE/_ref"
if [ ! -d "$SRC" ]; then
    echo "reference tree not found at $REF; skipping oracle/_ref build" >&2
    exit 0
fi
mkdir -p "$OUT"
INC="-I$HERE/ref_shim -I$SRC/BasicOperations -I$SRC/RiemannSolvers -I$SRC/Fluxes \
 -I$SRC/Integrators/DGSEMIntegrator -I$SRC/Integrators/Lifting -I$SRC/Integrators/Lifting/LiftingBR1 \
 -I$SRC/Integrators/BoundaryConditions -I$SRC/Indicators -I$SRC/ModalBasis -I$SRC/Physics"
FILES="$SRC/BasicOperations/BasicOperations.cpp $SRC/RiemannSolvers/ChandrashekarFlux.cpp \
 $SRC/Fluxes/NavierStokesFlux.cpp $SRC/Integrators/DGSEMIntegrator/DGSEMIntegrator.cpp \
 $SRC/Integrators/Lifting/LiftingScheme.cpp $SRC/Integrators/Lifting/LiftingBR1/LiftingBR1.cpp \
 $SRC/Indicators/Indicator.cpp $SRC/Indicators/PerssonPeraireIndicator.cpp $SRC/ModalBasis/ModalBasis.cpp \
 $SRC/Integrators/BoundaryConditions/BdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/SlipWallBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/SupersonicInflowBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SupersonicOutflowBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/SpecifiedStateBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/SymmetryBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SubsonicOutflowPBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/SubsonicInflowRVBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/SubsonicInflowPtTtAngBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/RiemannInvariantBdrFaceIntegrator.cpp \
 $SRC/Integrators/BoundaryConditions/NoSlipAdiabWallBdrFaceIntegrator.cpp $SRC/Integrators/BoundaryConditions/NoSlipIsothWallBdrFaceIntegrator.cpp \
 $HERE/ref_shim/ref_driver.cpp"
CXXFLAGS="-O2 -ffp-contract=off -std=c++17 -shared -fPIC -w"
g++ $CXXFLAGS $INC -DSUBCELL_FV_BLENDING $FILES -o "$OUT/libref_euler.so"
g++ $CXXFLAGS $INC -DPARABOLIC -DSUBCELL_FV_BLENDING $FILES -o "$OUT/libref_ns.so"
# where the tree was found, for the tests that read its mesh files
echo "$REF" > "$OUT/REFERENCE_TREE"
echo "built $OUT/libref_euler.so $OUT/libref_ns.so"
