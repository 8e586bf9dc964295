#!/bin/sh
# Recipe: compile the reference-built oracle (oracle/_ref/ref_driver) from the
# reference sources where they lie.  The checkout is taken from
# $RISGRAPH_REFERENCE, else from the location the reference is mounted at in
# the build container; without a checkout nothing is built (a GPU machine keeps
# the binaries it was given).  Test infrastructure only.
set -e
REF="${RISGRAPH_REFERENCE:-/root/reference}"
exec make -s -C "$(dirname "$0")" REF="$REF"
