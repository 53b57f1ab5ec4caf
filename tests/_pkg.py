"""Load the wfa2lib-rs_b200 package (its directory name is not an identifier)."""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load():
    if "wfa_b200" in sys.modules:
        return sys.modules["wfa_b200"]
    d = os.path.join(ROOT, "wfa2lib-rs_b200")
    spec = importlib.util.spec_from_file_location(
        "wfa_b200", os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wfa_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
