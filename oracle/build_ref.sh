#!/usr/bin/env bash
# Compile the reference's own CPU loops into oracle/_ref/libmgvref.so.
#
# Test infrastructure only (the oracle's pin).  The functions are taken at
# build time from the reference sources where they lie -- from
# "size_t stable_select_cpu" up to "hash_exchange" in src/main8.cu and
# src/main9.cu -- and piped straight into g++ together with ref_shim.cpp;
# no reference source is written into this repository.  Needs the
# reference checkout (default /root/reference, or $MGV_REFERENCE); without
# it the script exits 0 and prints why, and the prebuilt library (if any)
# is used as is.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${MGV_REFERENCE:-/root/reference}"
out="$here/_ref"
if [[ ! -f "$ref/src/main8.cu" || ! -f "$ref/src/main9.cu" ]]; then
    echo "build_ref: reference sources not found under $ref; skipping"
    exit 0
fi
mkdir -p "$out"
take() {
    awk '/^size_t stable_select_cpu/{p=1} /^vector<d_operator_t \*> hash_exchange/{p=0} p' "$1"
}
{
    echo '#include <cstdint>'
    echo '#include <cstddef>'
    echo 'namespace ref8 {'
    take "$ref/src/main8.cu"
    echo '}'
    echo 'namespace ref9 {'
    take "$ref/src/main9.cu"
    echo '}'
    cat "$here/ref_shim.cpp"
} | g++ -std=c++17 -O2 -fwrapv -shared -fPIC -x c++ - -o "$out/libmgvref.so"
echo "build_ref: wrote $out/libmgvref.so"
