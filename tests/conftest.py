import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, 'solfec-1.0_b200'), os.path.join(ROOT, 'oracle'), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built library')


_SCENES = {}


@pytest.fixture(scope='session')
def scene_cache():
    """Seeded scenes shared by the tests of one session (generation takes seconds)."""
    from solfec_b200 import scenes

    def get(name, **kw):
        key = (name, tuple(sorted(kw.items())))
        if key not in _SCENES:
            _SCENES[key] = getattr(scenes, name)(**kw)
        return _SCENES[key]
    return get
