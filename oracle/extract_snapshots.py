"""Extract the assembled GLSL fragment programs from the reference's snapshot file.

Test infrastructure for the oracle only (nothing in the product imports this).

The reference pins every generated program byte-for-byte in
``tests/compiler/__snapshots__/generated-glsl.snapshot.test.ts.snap`` (one vitest
``exports[...]`` entry per scene x strategy case, listed at
``tests/compiler/generated-glsl.snapshot.test.ts:58-110``).  Each entry is a
pretty-printed ``CompiledRenderer`` (``src/compiler/types.ts:1084-1136``) whose
``shaders["<id>-main"].fragment`` string is the whole transport program.  This
script pulls those strings out, undoes the template-literal escaping and writes
one ``.glsl`` file per case.
"""
import json
import os
import re
import sys

SNAP_REL = "tests/compiler/__snapshots__/generated-glsl.snapshot.test.ts.snap"

_ENTRY = re.compile(r"^exports\[`generated GLSL snapshot \(§2\.10 refactor safety net\) > (.*) 1`\] = `$")


def slug(name: str) -> str:
    return re.sub(r"[^a-z0-9]+", "_", name.lower()).strip("_")


def _unescape(s: str) -> str:
    # Template literal escaping used by vitest's snapshot serializer.
    return s.replace("\\`", "`").replace("\\${", "${").replace("\\\\", "\\")


def _renderer_meta(body):
    """The renderer's ``parameters`` and ``uniforms`` entries (defaults and the
    parameter paths each uniform is computed from), parsed from the pretty-printed
    object.  The ``shaders``/``sourceMaps``/``pipeline`` members are dropped first:
    only the two small tables are needed to bind uniforms."""
    text = _unescape("\n".join(body))
    out = {}
    for key in ("parameters", "uniforms"):
        m = re.search(r'^  "%s": ([\[{])$' % key, text, re.M)
        if not m:
            continue
        close = "]" if m.group(1) == "[" else "}"
        end = text.index("\n  " + close, m.end())
        chunk = m.group(1) + text[m.end():end] + "\n" + close
        chunk = chunk.replace("undefined", "null")
        chunk = re.sub(r",(\s*[}\]])", r"\1", chunk)
        out[key] = json.loads(chunk)
    return out


def extract(snap_path: str):
    """Yield (case_name, renderer_id, fragment_source, meta) for every snapshot case."""
    with open(snap_path, encoding="utf-8") as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines):
        m = _ENTRY.match(lines[i])
        if not m:
            i += 1
            continue
        name = m.group(1)
        j = i + 1
        while j < len(lines) and lines[j] != "`;":
            j += 1
        body = lines[i + 1:j]
        rid = None
        for ln in body:
            mm = re.match(r'^  "id": "(.*)",$', ln)
            if mm:
                rid = mm.group(1)
                break
        # Locate "<id>-main": { ... "fragment": "<source>",   "vertex": ...
        frag = None
        for k, ln in enumerate(body):
            if rid is not None and ln.strip() == f'"{rid}-main": {{':
                fl = body[k + 1]
                assert fl.lstrip().startswith('"fragment": "'), fl
                src = [fl.lstrip()[len('"fragment": "'):]]
                q = k + 2
                while not (body[q - 1].endswith('",') and body[q].lstrip().startswith('"vertex": "')):
                    src.append(body[q])
                    q += 1
                text = "\n".join(src)
                assert text.endswith('",')
                frag = _unescape(text[:-2])
                break
        if frag is not None:
            yield name, rid, frag, _renderer_meta(body)
        i = j + 1


def main(argv):
    ref_root = argv[1]
    out_dir = argv[2]
    os.makedirs(out_dir, exist_ok=True)
    index = {}
    for name, rid, frag, meta in extract(os.path.join(ref_root, SNAP_REL)):
        fn = slug(name) + ".glsl"
        with open(os.path.join(out_dir, fn), "w", encoding="utf-8") as f:
            f.write(frag)
        index[slug(name)] = {"case": name, "renderer": rid, "file": fn, **meta}
    with open(os.path.join(out_dir, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)
    print(f"extracted {len(index)} programs into {out_dir}")


if __name__ == "__main__":
    main(sys.argv)
