"""Location of an XCALibre.jl checkout for the tests that read its grid files
in place (the committed fixtures under tests/golden/ cover the same data).

Set XCAL_REFERENCE_DIR to the checkout's root; when it is unset, ref_path()
returns "" and those tests skip.
"""
import os

REF_DIR = os.environ.get("XCAL_REFERENCE_DIR", "")


def ref_path(*parts: str) -> str:
    """Path inside the checkout, or "" when XCAL_REFERENCE_DIR is unset."""
    return os.path.join(REF_DIR, *parts) if REF_DIR else ""
