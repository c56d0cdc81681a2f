"""Stencils the reference's frontend must reject are rejected here too.

``tests/golden/ref_rejects.json`` holds every ``@stencil`` definition that a
reference test wraps in ``pytest.raises(..., match=...)`` (extracted by
``tests/golden/make_golden.py``); decorating it with this package's
``stencil`` must raise with the same message fragment.
"""

import json
import os

import pytest

import ref_corpus as RC

with open(os.path.join(RC.GOLDEN, "ref_rejects.json")) as _f:
    _REJECTS = json.load(_f)


@pytest.mark.parametrize("key", sorted(_REJECTS))
def test_frontend_rejects_like_the_reference(tmp_path, key):
    e = _REJECTS[key]
    with pytest.raises(Exception, match=e["match"]):
        RC.build(tmp_path, key, e)
