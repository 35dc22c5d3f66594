"""Generate the loader fixture (loaders_golden.npz) by running the reference's
field-map loaders (src/PyPATools/field_src/field_loaders.py) on the synthetic
files of loader_files.write_cases, and its Field.from_file (field.py:284-343)
on each of them.

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden_loaders.py
"""
import contextlib
import io
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402
from loader_files import write_cases  # noqa: E402

LOADER = {"opera3d": "load_opera_table", "opera2d": "load_opera_table", "opera_e": "load_opera_table",
          "opera_ext": "load_opera_table", "comsol3d": "load_comsol", "comsol2d": "load_comsol",
          "opal": "load_opal_midplane", "opal_cut": "load_opal_midplane", "opal_cyl": "load_opal_midplane",
          "aima": "load_aima_agora", "aima_mirror": "load_aima_agora"}


def main():
    load_reference()
    from PyPATools.field_src import field_loaders
    from PyPATools import field
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (path, kwargs) in write_cases(tmp).items():
            with contextlib.redirect_stdout(io.StringIO()):
                data = getattr(field_loaders, LOADER[name])(path, **kwargs)
            for k, v in data["grid"].items():
                out[f"{name}/grid/{k}"] = np.asarray(v)
            for k, v in data["values"].items():
                out[f"{name}/values/{k}"] = np.asarray(v)
            out[f"{name}/dim"] = np.int64(data["dim"])
            out[f"{name}/field_type"] = np.array(data["field_type"])
            n = data["metadata"].get("n_points", {})
            for k, v in n.items():
                out[f"{name}/n_points/{k}"] = np.int64(v)
            # the reference's Field.from_file on the same file (default loader arguments)
            if not kwargs:
                try:
                    with contextlib.redirect_stdout(io.StringIO()):
                        f = field.Field.from_file(path)
                    out[f"{name}/from_file_dim"] = np.int64(f.dim)
                except Exception as exc:
                    out[f"{name}/from_file_error"] = np.array(type(exc).__name__)
            print(name, data["dim"], {k: np.shape(v) for k, v in data["values"].items()})
        # error cases
        bad = Path(tmp) / "mixed.table"
        bad.write_text("2 1 1\n1 X [cm]\n2 BX [T]\n3 EX [V/m]\n0\n0 1 2\n1 1 2\n")
        try:
            field_loaders.load_opera_table(str(bad))
        except Exception as exc:
            out["errors/opera_mixed"] = np.array(f"{type(exc).__name__}: {exc}")
    dest = HERE / "loaders_golden.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, dest.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
