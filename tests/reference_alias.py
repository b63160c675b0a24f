"""pytest plugin: makes `roughpy.compute` resolve to `roughpy_b200.compute`.

Loaded with `-p tests.reference_alias` when the reference's own compute test
files are run, unmodified, against the drop-in: they import
`from roughpy import compute` or `import roughpy.compute as rpc`, and this
plugin installs a `roughpy` package whose `compute` is the drop-in module
before they are collected.  Nothing of the reference is imported."""
import sys
import types


def pytest_configure(config):
    import roughpy_b200.compute as drop_in
    pkg = types.ModuleType("roughpy")
    pkg.__path__ = []
    pkg.compute = drop_in
    sys.modules["roughpy"] = pkg
    sys.modules["roughpy.compute"] = drop_in
