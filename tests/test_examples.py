"""The Python usage examples of the integration guide (section 4) run as
written, on a B200.  The test reads the guide itself on purpose: the code
blocks a user copies are the thing under test, so a copy kept elsewhere
could drift from them unnoticed."""
import re

import numpy as np
import pytest

from conftest import ROOT


@pytest.mark.gpu
def test_integration_python_examples_run():
    guide = f"{ROOT}/INTEGRATION.md"
    text = open(guide).read()
    sec = text[text.index("## 4. Python"):text.index("## 5.")]
    code = re.findall(r"```python\n(.*?)```", sec, flags=re.S)
    assert code
    env = {}
    exec(compile(code[0], guide, "exec"), env)
    assert env["stats"].max_div < 1e-5 and env["stats"].nan_detected == 0
    assert np.isfinite(env["U"]).all()
    c = env["concentration"]
    assert c.max() > 0 and np.isfinite(c).all()
    env["d"].close()
    env["p"].close()
