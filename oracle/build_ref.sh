#!/usr/bin/env bash
# Build the reference oracle from the UNMODIFIED reference sources.
#
# TEST INFRASTRUCTURE ONLY.  For each NCOL given (default: 2 3 4) this
#   1. mirrors 4d_Q16/{include,susy,generic,libraries} as a symlink farm under
#      oracle/_ref/n<NCOL>/ -- every file is a symlink to the reference except
#      include/susy.h, which is regenerated with "#define NCOL <NCOL>" exactly
#      as the reference's own testsuite/scalar/run_tests:11 sed-edits it;
#   2. compiles the susy_hmc object set (susy/Make_template:155-159 plus the
#      MY_OBJECTS/G_OBJECTS lists) and the complex/susy library routines with
#      the reference's flags (susy/Make_scalar:7, libraries/Make_vanilla:9),
#      plus -fPIC, linking oracle/lapack_min.c in place of -llapack -lblas;
#   3. links oracle/_ref/n<NCOL>/susy_hmc (the reference program itself) and
#      oracle/_ref/libsusyref_n<NCOL>.so (reference objects minus control.o,
#      plus oracle/ref_harness.c) for ctypes.
# An argument <NCOL>smd builds the same with -DSMD_ALGORITHM added
# (the defines of susy/Make_template:112-116, target susy_smd) into
# oracle/_ref/n<NCOL>smd/ and libsusyref_n<NCOL>_smd.so.  Not built by
# default: that build's pseudofermion refresh reads uninitialised memory
# (grsource.c:79-92) and printed NaN actions on its first trajectory here,
# so it cannot serve as an oracle.
# An argument shim<NCOL> (after <NCOL> in the same call or an earlier one)
# links the reference's susy_hmc once more with susy_b200/shim/b200_shim.c
# in place of the hot-path functions it replaces, against
# susy_b200/libsusy_b200.so: the replaced symbols are weakened in copies of
# the reference objects (objcopy --weaken-symbol), so the shim's strong
# definitions win at link time; output oracle/_ref/n<NCOL>/susy_hmc_b200.
# Arguments cheb<NCOL> and mode<NCOL> build the reference's susy_cheb and
# susy_mode (chebyshev.c and modenumber.c call DSq and congrad_multi), each
# plain and with the shim, into oracle/_ref/n<NCOL>cheb/ and n<NCOL>mode/.
# Outputs go only to oracle/_ref/ (git-ignored, shipped with the tree).
# The reference's own build system is not used.
set -euo pipefail

REF=${SUSY_REFERENCE:-/root/reference}/4d_Q16
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
CC=${CC:-gcc}
JOBS=${JOBS:-8}

if [ ! -d "$REF/susy" ]; then
  echo "build_ref.sh: reference sources not found at $REF" >&2
  exit 2
fi

NCOLS=("$@")
[ ${#NCOLS[@]} -eq 0 ] && NCOLS=(2 3 4)

MY_OBJECTS="setup setup_lambda setup_offset action plaq ploop unit scalar_eig
            link_trace widths determinant grsource utilities library_util
            gauge_info congrad_multi"
HMC_OBJECTS="update_o update_h setup_rhmc det_force"
G_OBJECTS="io_helpers io_lat io_lat_utils make_lattice nersc_cksum ranstuff
           gaugefix remap_stdio_from_args layout_hyper_prime io_ansi com_vanilla"
LIB_OBJECTS="cmplx cexp clog csqrt ce_itheta dcmplx dcexp dclog dcsqrt dce_itheta
             cmp_ahmat dump_ahmat make_ahmat uncmp_ahmat rand_ahmat
             m_su2_mat_vec_n m_su2_mat_vec_a gaussrand z2rand byterevn m_mat_an
             m_mat_na m_mat_nn realtr s_m_a_mat s_m_a_amat s_m_s_mat s_m_s_amat
             adjoint mat_copy trace complextr dumpmat dumpsu2 clear_mat addmat
             addamat submat subamat clearvec r_su2_hit_a l_su2_hit_n s_m_mat
             s_m_amat s_a_d_mat cs_a_d_mat s_m_mat_nn s_m_mat_na s_m_mat_an
             cs_m_mat cs_m_a_mat cs_m_a_amat cs_m_a_mata cs_m_s_mat"

APP_FLAGS="-O3 -DP4 -Wall -fno-strict-aliasing -fPIC -DSINGLE -DPRECISION=2
           -D_FILE_OFFSET_BITS=64 -D_LARGEFILE_SOURCE64
           -DPHI_ALGORITHM -DHMC_ALGORITHM -w"
LIB_FLAGS="-O3 -Wall -fPIC -DPRECISION=2 -w"

# symlink farm of the reference sources under $1 with NCOL = $2
farm() {
  local D=$1 N=$2
  mkdir -p "$D/obj"
  for sub in include susy generic libraries; do
    mkdir -p "$D/$sub"
    for f in "$REF/$sub"/*.c "$REF/$sub"/*.h; do
      [ -e "$f" ] || continue
      local b
      b=$(basename "$f")
      [ "$sub/$b" = "include/susy.h" ] && continue
      ln -sf "$f" "$D/$sub/$b"
    done
  done
  sed -E "s/^(#define NCOL) .*/\1 $N/" "$REF/include/susy.h" > "$D/include/susy.h.tmp"
  if ! cmp -s "$D/include/susy.h.tmp" "$D/include/susy.h" 2>/dev/null; then
    mv "$D/include/susy.h.tmp" "$D/include/susy.h"
  else
    rm -f "$D/include/susy.h.tmp"
  fi
}

# compile src to out with flags unless out is newer than src and susy.h of $D
compile() {   # src out flags...
  local src=$1 out=$2
  shift 2
  if [ ! -e "$out" ] || [ "$src" -nt "$out" ] || [ "$D/include/susy.h" -nt "$out" ]; then
    $CC -c "$@" "$src" -o "$out"
  fi
}

build_one() {
  local N=${1%smd}
  local ALG=-DHMC_ALGORITHM SUF=""
  if [ "$1" != "$N" ]; then ALG="-DHMC_ALGORITHM -DSMD_ALGORITHM"; SUF=_smd; fi
  local D=$OUT/n$1
  local APP_FLAGS="${APP_FLAGS/-DHMC_ALGORITHM/$ALG}"
  farm "$D" "$N"

  local objs=() pids=()
  for o in $MY_OBJECTS $HMC_OBJECTS; do
    compile "$D/susy/$o.c" "$D/obj/$o.o" $APP_FLAGS -I"$D/susy" &
    objs+=("$D/obj/$o.o")
  done
  for o in $G_OBJECTS; do
    compile "$D/generic/$o.c" "$D/obj/g_$o.o" $APP_FLAGS -I"$D/susy" &
    objs+=("$D/obj/g_$o.o")
  done
  for o in $LIB_OBJECTS; do
    compile "$D/libraries/$o.c" "$D/obj/l_$o.o" $LIB_FLAGS &
    objs+=("$D/obj/l_$o.o")
  done
  compile "$D/susy/control.c" "$D/obj/control.o" $APP_FLAGS -I"$D/susy" &
  compile "$HERE/lapack_min.c" "$D/obj/lapack_min.o" -O2 -fPIC -Wall &
  # The harness is project code compiled against the reference headers
  ln -sf "$HERE/ref_harness.c" "$D/susy/zz_ref_harness.c"
  compile "$D/susy/zz_ref_harness.c" "$D/obj/ref_harness.o" $APP_FLAGS -I"$D/susy" &
  wait

  $CC -o "$D/susy_hmc" "$D/obj/control.o" "${objs[@]}" "$D/obj/lapack_min.o" -lm
  $CC -shared -o "$OUT/libsusyref_n$N$SUF.so" "$D/obj/ref_harness.o" "${objs[@]}" \
      "$D/obj/lapack_min.o" -lm
  echo "built $D/susy_hmc and $OUT/libsusyref_n$N$SUF.so"
}

# Link $D/<control>'s program once more with the shim: fermion_op / DSq
# (utilities.c), congrad_multi, and -- where the program has them --
# fermion_force and gauge_force (update_h.c) and update_u (update_o.c) are
# taken from susy_b200/shim/b200_shim.c.  $1 = object dir root, $2 = its
# control object, $3 = output program, $4 = the APP_FLAGS it was built with
link_shim() {
  local D=$1 CTRL=$2 PROG=$3 FLAGS=$4
  local ROOT
  ROOT=$(cd "$HERE/.." && pwd)
  if [ ! -e "$ROOT/susy_b200/libsusy_b200.so" ]; then
    echo "build_ref.sh: susy_b200/libsusy_b200.so not built" >&2
    exit 2
  fi
  mkdir -p "$D/objw"
  objcopy --weaken-symbol=fermion_op --weaken-symbol=DSq "$D/obj/utilities.o" "$D/objw/utilities.o"
  objcopy --weaken-symbol=congrad_multi "$D/obj/congrad_multi.o" "$D/objw/congrad_multi.o"
  [ -e "$D/obj/update_h.o" ] && objcopy --weaken-symbol=fermion_force \
      --weaken-symbol=gauge_force "$D/obj/update_h.o" "$D/objw/update_h.o"
  [ -e "$D/obj/update_o.o" ] && objcopy --weaken-symbol=update_u "$D/obj/update_o.o" \
      "$D/objw/update_o.o"
  ln -sf "$ROOT/susy_b200/shim/b200_shim.c" "$D/susy/zz_b200_shim.c"
  $CC -c $FLAGS -I"$D/susy" -I"$ROOT/include" "$D/susy/zz_b200_shim.c" -o "$D/objw/b200_shim.o"
  local objs=()
  for f in "$D"/obj/*.o; do
    local b
    b=$(basename "$f")
    case "$b" in
      control*.o|ref_harness.o|lapack_min.o) continue ;;
      utilities.o|congrad_multi.o|update_h.o|update_o.o) objs+=("$D/objw/$b") ;;
      *) objs+=("$f") ;;
    esac
  done
  $CC -o "$D/$PROG" "$D/obj/$CTRL" "${objs[@]}" "$D/objw/b200_shim.o" \
      "$D/obj/lapack_min.o" -L"$ROOT/susy_b200" -lsusy_b200 \
      -Wl,-rpath,'$ORIGIN/../../../susy_b200' -lm
  echo "built $D/$PROG"
}

build_shim() {
  local N=$1 D=$OUT/n$1
  if [ ! -e "$D/obj/utilities.o" ]; then
    echo "build_ref.sh: build NCOL=$N before shim$N" >&2
    exit 2
  fi
  link_shim "$D" control.o susy_hmc_b200 "$APP_FLAGS"
}

# The reference's measurement programs that call the hot path
# (susy/Make_template:152-162): susy_cheb (chebyshev.c:45,60 call DSq)
# and susy_mode (modenumber.c:26,63,66 call congrad_multi), each with its
# own defines and objects, plain and with the shim, into
# oracle/_ref/n<NCOL><name>/susy_<name>[_b200].
build_app() {
  local N=$1 NAME=$2 DEFS=$3 EXTRA=$4 CTRL=$5
  D=$OUT/n$N$NAME
  local FLAGS="${APP_FLAGS/-DHMC_ALGORITHM/$DEFS}"
  farm "$D" "$N"
  local objs=()
  for o in $MY_OBJECTS $EXTRA; do
    compile "$D/susy/$o.c" "$D/obj/$o.o" $FLAGS -I"$D/susy" &
    objs+=("$D/obj/$o.o")
  done
  for o in $G_OBJECTS; do
    compile "$D/generic/$o.c" "$D/obj/g_$o.o" $FLAGS -I"$D/susy" &
    objs+=("$D/obj/g_$o.o")
  done
  for o in $LIB_OBJECTS; do
    compile "$D/libraries/$o.c" "$D/obj/l_$o.o" $LIB_FLAGS &
    objs+=("$D/obj/l_$o.o")
  done
  compile "$HERE/lapack_min.c" "$D/obj/lapack_min.o" -O2 -fPIC -Wall &
  wait
  local plain=()
  for f in "${objs[@]}"; do
    [ "$(basename "$f")" = "$CTRL" ] || plain+=("$f")
  done
  $CC -o "$D/susy_$NAME" "$D/obj/$CTRL" "${plain[@]}" "$D/obj/lapack_min.o" -lm
  echo "built $D/susy_$NAME"
  link_shim "$D" "$CTRL" "susy_${NAME}_b200" "$FLAGS"
}

mkdir -p "$OUT"
for N in "${NCOLS[@]}"; do
  case "$N" in
    shim*) build_shim "${N#shim}" ;;
    cheb*) build_app "${N#cheb}" cheb "-DPHI_ALGORITHM -DCHEB -DRESCALE" \
               "control_cheb chebyshev z2source" control_cheb.o ;;
    mode*) build_app "${N#mode}" mode "-DPHI_ALGORITHM -DMODE -DRESCALE" \
               "control_mode modenumber mode_coeffs z2source" control_mode.o ;;
    *) build_one "$N" ;;
  esac
done
