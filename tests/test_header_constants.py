"""The C header's enums (include/hedge_b200.h) and the Python layer's and
the oracle's copies of them agree: model ids, precisions, boundary kinds
and status codes."""
import os
import re

import hedge_b200.models as models
from hedge_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "hedge_b200.h")


def _enum(prefix):
    text = open(HEADER).read()
    return {m.group(1): int(m.group(2))
            for m in re.finditer(r"\b%s_(\w+)\s*=\s*(\d+)" % prefix, text)}


def test_models():
    hdr = _enum("HB_MODEL")
    assert hdr and all(getattr(models, "MODEL_" + k) == v for k, v in hdr.items())


def test_boundary_kinds():
    hdr = _enum("HB_BC")
    assert "INCIDENT" in hdr
    assert all(getattr(models, "BC_" + k) == v for k, v in hdr.items())
    import oracle
    assert all(getattr(oracle, "BC_" + k) == v for k, v in hdr.items())


def test_precisions_and_status():
    prec = _enum("HB_PREC")
    assert all(getattr(_native, "PREC_" + k) == v for k, v in prec.items())
    st = _enum("HB_ERR")
    assert all(getattr(_native, "HB_ERR_" + k) == v for k, v in st.items())
