"""Import helper: load the ``mbd-icenav_b200`` directory as package ``mbd_icenav_b200``."""
import importlib.util
import os
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))


def load_package():
    if "mbd_icenav_b200" in sys.modules:
        return sys.modules["mbd_icenav_b200"]
    spec = importlib.util.spec_from_file_location(
        "mbd_icenav_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mbd_icenav_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
