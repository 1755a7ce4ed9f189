"""Where the tests find the reference tree: the environment variable
ICEMPM_REFERENCE, else the reference's location in the build container.
Tests that read the reference tree skip where it is absent (the GPU box); the
committed fixtures under tests/golden/ stand in for it there."""
import os

REF = os.environ.get("ICEMPM_REFERENCE", "/root/reference")
GEOM = os.path.join(REF, "build", "geometries_2d")
INPUTS = os.path.join(REF, "input_")
BUILD_JSON = os.path.join(REF, "build")
