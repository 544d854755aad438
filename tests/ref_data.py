"""The reference's own seed sets (data/100K-{blue,white,perturbed-grid}.xyz,
README.md:15-25), stored unchanged as xz fixtures by
tests/golden/make_ref_data.py and read through the library's seed loader.

CAPS are the caps the reference's README runs each set with."""
import lzma
import os
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("blue", "white", "perturbed-grid")
CAPS = {"blue": dict(K=20, P=25, V=30), "perturbed-grid": dict(K=50, P=30, V=40), "white": dict(K=70, P=30, V=40)}
COUNT = 97336


def fixture_path(name):
    return os.path.join(HERE, "golden", f"ref_data_100k-{name}.xyz.xz")


def text(name) -> bytes:
    with lzma.open(fixture_path(name), "rb") as f:
        return f.read()


def load(name):
    """(97336, 4) float32 seeds (w = 0) through rpd.load_seeds."""
    import rpd

    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, f"100K-{name}.xyz")
        with open(p, "wb") as f:
            f.write(text(name))
        return rpd.load_seeds(p)
