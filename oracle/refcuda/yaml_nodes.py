"""ORACLE BUILD SHIM — test infrastructure, not product code.

Writes the node tree of a YAML file, as composed by PyYAML, next to it
(`<path>.nodes`), for the yaml-cpp stand-in the reference CUDA build links
(oracle/refcuda/shim/yaml_shim.cpp documents the format). Composition keeps
complex keys (a flow sequence such as `[J: 1, P: -1]` used as a mapping key)
and document order, as yaml-cpp does.

Usage: python -m oracle.refcuda.yaml_nodes config.yml [more.yml ...]
"""
import sys

import yaml

_NULL = "tag:yaml.org,2002:null"


def _emit(node, out):
    if isinstance(node, yaml.ScalarNode):
        if node.tag == _NULL:
            out.append(b"N\n")
        else:
            b = node.value.encode("utf-8")
            out.append(b"S %d\n" % len(b) + b + b"\n")
    elif isinstance(node, yaml.SequenceNode):
        out.append(b"Q %d\n" % len(node.value))
        for v in node.value:
            _emit(v, out)
    elif isinstance(node, yaml.MappingNode):
        out.append(b"M %d\n" % len(node.value))
        for k, v in node.value:
            _emit(k, out)
            _emit(v, out)
    else:
        raise TypeError(f"unexpected YAML node {type(node).__name__}")


def write_nodes(path):
    """Compose `path` with PyYAML and write `path + '.nodes'`."""
    with open(path, "rb") as f:
        root = yaml.compose(f)
    out = []
    _emit(root if root is not None else yaml.ScalarNode(_NULL, ""), out)
    with open(str(path) + ".nodes", "wb") as f:
        f.write(b"".join(out))
    return str(path) + ".nodes"


if __name__ == "__main__":
    for p in sys.argv[1:]:
        print(write_nodes(p))
