"""Writes tests/golden/params_ref.json: the reference's own SimParams::Reset
and SimParams::ParseFile (oracle/_ref/libref_params.so, built by
oracle/Makefile from the reference's parameters_sim.cpp, which needs the
rapidjson headers named by RAPIDJSON_INC) applied to the parameter files of
the reference tree and to the test configurations of tests/test_capi_host.py.

For each case the file holds the JSON text, the parser's return code, the
"InputRawPoints" string and the resulting icy::SimParams as hex bytes, so
the project's parser can be pinned to the reference's where neither the
reference tree nor rapidjson is present.

    RAPIDJSON_INC=<dir holding rapidjson/> make -C oracle ref
    python tests/golden/make_params_golden.py
"""
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    from oracle.oracle import RefParams
    from refpaths import BUILD_JSON, INPUTS
    from test_capi_host import CONFIGS
    R = RefParams()
    cases = []
    texts = []
    for d in (INPUTS, BUILD_JSON):
        for name in sorted(os.listdir(d)):
            if name.endswith(".json"):
                texts.append((os.path.relpath(os.path.join(d, name), os.path.dirname(d)),
                              open(os.path.join(d, name)).read()))
    for k, cfg in enumerate(CONFIGS):
        texts.append((f"test_config_{k}", json.dumps(cfg, indent=1)))
    with tempfile.TemporaryDirectory() as tmp:
        for name, text in texts:
            path = os.path.join(tmp, "cfg.json")
            with open(path, "w") as f:
                f.write(text)
            p = R.reset()
            rc, raw, _ = R.parse_file(p, path)
            cases.append({"name": name, "text": text, "rc": rc, "raw": raw, "params": bytes(p).hex()})
    out = {"reset": bytes(R.reset()).hex(), "cases": cases}
    with open(os.path.join(HERE, "params_ref.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(len(cases), "cases")


if __name__ == "__main__":
    main()
