#!/usr/bin/env bash
# Generates the compile-time configuration header for the GR-Athena++ reference
# build used as the parity oracle (test infrastructure only).
#
# The reference normally produces src/defs.hpp with its own configure script.
# That script is not run here: this recipe fills the template's @KEY@ slots
# (src/defs.hpp.in) with the values that `-z -z_vc --nghost=4 -omp` selects,
# and writes the result into the git-ignored build folder.  Nothing from the
# reference is copied into the repository.
#
# usage: mkdefs.sh <reference root> <output header> <problem name>
set -euo pipefail
REF="$1"
OUT="$2"
PROB="${3:-z4c_oracle_pgen}"

sed \
  -e 's|@GIT_HASH@|oracle-build|' \
  -e 's|@DBG_FALLBACK_NO_TABLE_LIMITS@|NO_DBG_FALLBACK_NO_TABLE_LIMITS|' \
  -e "s|@PROBLEM@|${PROB}|" \
  -e 's|@COORDINATE_SYSTEM@|cartesian|' \
  -e 's|@FLUID_ENABLED@|0|' \
  -e 's|@HYBRID_INTERP@|NO_HYBRID_INTERP|' \
  -e 's|@EQUATION_OF_STATE@|none|' \
  -e 's|@EOS_POLICY@||' \
  -e 's|@COLDEOS_POLICY@||' \
  -e 's|@EOS_POLICY_CODE@|0|' \
  -e 's|@ERROR_POLICY@||' \
  -e 's|@ERROR_POLICY_CODE@|0|' \
  -e 's|@PRIMITIVE_SOLVER_ADJUST_CONSERVED@|PRIMITIVE_SOLVER_ADJUST_CONSERVED|' \
  -e 's|@MAGNETIC_FIELDS_ENABLED@|0|' \
  -e 's|@GENERAL_RELATIVITY@|0|' \
  -e 's|@Z4C_ENABLED@|1|' \
  -e 's|@CCE_ENABLED@|0|g' \
  -e 's|@WAVE_ENABLED@|0|' \
  -e 's|@WAVE_CC_ENABLED@|0|' \
  -e 's|@WAVE_CX_ENABLED@|0|' \
  -e 's|@WAVE_VC_ENABLED@|0|' \
  -e 's|@Z4C_CC_ENABLED@|NO_Z4C_CC_ENABLED|' \
  -e 's|@Z4C_CX_ENABLED@|NO_Z4C_CX_ENABLED|' \
  -e 's|@Z4C_VC_ENABLED@|Z4C_VC_ENABLED|' \
  -e 's|@Z4C_CX_NUM_RBC@|0|' \
  -e 's|@Z4C_CX_NUM_RBC_INIT_LO@|Z4C_CX_NUM_RBC_INIT_LO|' \
  -e 's|@Z4C_WITH_HYDRO_ENABLED@|NO_Z4C_WITH_HYDRO_ENABLED|' \
  -e 's|@M1_ENABLED@|0|' \
  -e 's|@M1_BNS_NURATES@|0|' \
  -e 's|@EJECTA_ENABLED@|NO_EJECTA_ENABLED|' \
  -e 's|@SINGLE_PRECISION_ENABLED@|0|' \
  -e 's|@H5_DOUBLE_PRECISION_ENABLED@|0|' \
  -e 's|@TWO_PUNCTURES_OPTION@|NO_TWO_PUNCTURES|' \
  -e 's|@LORENE_OPTION@|NO_LORENE|' \
  -e 's|@LORENE_HARDCODED_UNITS@|NO_LORENE_HARDCODED_UNITS|' \
  -e 's|@Z4C_ETA_CONF@|NO_Z4C_ETA_CONF|' \
  -e 's|@Z4C_ETA_TRACK_TP@|NO_Z4C_ETA_TRACK_TP|' \
  -e 's|@Z4C_REF_BOX_IN_BOX@|Z4C_REF_BOX_IN_BOX|' \
  -e 's|@Z4C_REF_SPHERES@|NO_Z4C_REF_SPHERES|' \
  -e 's|@MPI_OPTION@|NOT_MPI_PARALLEL|' \
  -e 's|@MPI_NO_PERSIST_OPTION@|NO_MPI_NO_PERSIST|' \
  -e 's|@OPENMP_OPTION@|OPENMP_PARALLEL|' \
  -e 's|@HDF5_OPTION@|NO_HDF5OUTPUT|' \
  -e 's|@GSL_OPTION@|NO_GSL|' \
  -e 's|@DEBUG_OPTION@|NOT_DEBUG|' \
  -e 's|@EXCEPTION_HANDLING_OPTION@|ENABLE_EXCEPTIONS|' \
  -e 's|@COMPILER_CHOICE@|g++|' \
  -e 's|@COMPILER_COMMAND@|g++|' \
  -e 's|@COMPILER_FLAGS@|oracle recipe|' \
  -e 's|@NHYDRO_VARIABLES@|0|' \
  -e 's|@NFIELD_VARIABLES@|0|' \
  -e 's|@NWAVE_VALUE@|5|' \
  -e 's|@NUMBER_PASSIVE_SCALARS@|0|' \
  -e 's|@NUMBER_GHOST_CELLS@|4|' \
  -e 's|@NUMBER_COARSE_GHOSTS@|4|' \
  -e 's|@NUMBER_COARSE_GHOSTS_CX@|4|' \
  -e 's|@NUMBER_EXTRAPOLATION_POINTS@|5|' \
  -e 's|@NUMBER_INTERP_GHOSTS@|2|' \
  "${REF}/src/defs.hpp.in" > "${OUT}.tmp"

if grep -n '@[A-Z0-9_]*@' "${OUT}.tmp"; then
  echo "mkdefs.sh: unfilled template slots remain" >&2
  exit 1
fi
mv "${OUT}.tmp" "${OUT}"
