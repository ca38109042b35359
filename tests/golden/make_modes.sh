#!/bin/sh
# Regenerates tests/golden/modes/*.txt.gz with the reference's own Arnoldi mode
# solver (oracle/_ref/modegen, built by `make -C oracle ref`) and records the
# solver's beta for each in modes/betas.txt.  Arguments: window nx ny, disc
# (um), core [left,right) x [bottom,top), ep_clad, ep_core, wavelength (um),
# Krylov size, tolerance.  Takes a few minutes on one core.
set -e
here=$(cd "$(dirname "$0")" && pwd)
gen="$here/../../oracle/_ref/modegen"
cd "$here/modes"
: > betas.txt
run() {
    name=$1; shift
    "$gen" "$@" "$name.txt" 2> "$name.log"
    printf '%s %s\n' "$name" "$(grep 'modegen: beta' "$name.log" | sed 's/.*beta = //; s/ *n_eff.*//')" >> betas.txt
    rm -f "$name.log"
}
# 500 x 250 nm strip on a 0.05 um grid (small test problems)
run small_te0 24 16 0.05 7 17 6 11 2.085 12.1 1.55 20 1e-5
# 500 x 225 nm input end and 3.0 um x 225 nm output end of the 200x160x400 taper, 0.025 um grid
run c1_in_te0 64 48 0.025 22 42 20 29 2.085 12.1 1.55 20 1e-5
run c1_out_te0 160 48 0.025 20 140 20 29 2.085 12.1 1.55 20 1e-5
gzip -9 -f small_te0.txt c1_in_te0.txt c1_out_te0.txt
