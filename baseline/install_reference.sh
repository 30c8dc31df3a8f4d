#!/usr/bin/env bash
# Install the unmodified reference package (accusim, pure Python) into baseline/_ref.
#
# The GPU plug-ins subclass accusim's own Force and Integrator classes, the tests run them inside
# accusim's Simulation.run, and `bench.py --impl reference` times accusim's NumPy path, so the
# reference must be importable wherever those run. baseline/_ref is git-ignored but travels with the
# working tree. Offline install: no index, no dependency resolution (numpy and scipy are already in
# the environment). The source is copied first because setuptools writes build files next to it.
#
#   ACCUSIM_SRC=/path/to/DevinProj bash baseline/install_reference.sh
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
src="${ACCUSIM_SRC:?set ACCUSIM_SRC to a checkout of the reference (the directory holding pyproject.toml)}"
tmp="$(mktemp -d)"
trap 'rm -rf "$tmp"' EXIT
cp -r "$src"/. "$tmp"/
rm -rf "$tmp/build"
python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
    --target "$here/_ref" --upgrade "$tmp"
python - "$here/_ref" <<'EOF'
import sys
sys.path.insert(0, sys.argv[1])
import accusim
print("accusim", accusim.__file__)
EOF
