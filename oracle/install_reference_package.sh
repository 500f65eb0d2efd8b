#!/bin/sh
# Installs the reference's own Python package (python/apocharmm, pure ctypes
# over the C ABI, unmodified) into baseline/_ref, which travels to the GPU
# machines with the repository but stays out of its history.  The package
# has no packaging metadata of its own, so the install runs from a copy
# under /tmp given a minimal pyproject.toml; none of its files change.
#   REF=<reference sources> sh oracle/install_reference_package.sh
set -e
REF=${REF:-${APOCHARMM_REFERENCE_SOURCES:-/root/reference}}
ROOT=$(cd "$(dirname "$0")/.." && pwd)
TMP=$(mktemp -d /tmp/apo_refpkg.XXXXXX)
cp -r "$REF/python/apocharmm" "$TMP/apocharmm"
cat > "$TMP/pyproject.toml" <<'TOML'
[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"
[project]
name = "apocharmm"
version = "0.0.0"
[tool.setuptools]
packages = ["apocharmm"]
TOML
python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
  --target "$ROOT/baseline/_ref" --upgrade "$TMP"
rm -rf "$TMP"
