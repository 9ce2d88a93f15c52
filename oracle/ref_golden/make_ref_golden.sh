#!/bin/sh
# Pin the oracle to the reference crate's own outputs where a Rust toolchain
# exists (none does on the machines this repository was built on).
#   1. python tests/golden/make_ref_inputs.py   (writes tests/golden/ref_inputs.txt)
#   2. sh oracle/ref_golden/make_ref_golden.sh [path of the reference crate]
# builds a small program against the reference crate's sources, in
# oracle/_ref/ref_golden (git-ignored), runs it on the inputs and writes
# tests/golden/ref_prices.txt, which tests/test_oracle.py then compares with
# the oracle bit for bit.  Needs cargo and the crate's dependencies in the
# local cargo registry (the build runs --offline).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/../.." && pwd)
REF=${1:-/root/reference}
if ! command -v cargo >/dev/null 2>&1; then
    echo "cargo not found: the reference crate cannot be built here; nothing written" >&2
    exit 2
fi
OUT="$ROOT/oracle/_ref/ref_golden"
mkdir -p "$OUT/src"
cp "$HERE/main.rs" "$OUT/src/main.rs"
cat > "$OUT/Cargo.toml" <<TOML
[package]
name = "ope_ref_golden"
version = "0.1.0"
edition = "2021"

[dependencies]
options_pricing_engine = { path = "$REF" }

[profile.release]
opt-level = 3
TOML
cargo build --release --offline --manifest-path "$OUT/Cargo.toml" --target-dir "$OUT/target"
"$OUT/target/release/ope_ref_golden" < "$ROOT/tests/golden/ref_inputs.txt" > "$ROOT/tests/golden/ref_prices.txt"
echo "wrote tests/golden/ref_prices.txt"
