"""The C-ABI library builds, loads and exports every entry point declared in
include/sawsim_b200.h (no compute calls: no GPU needed)."""
import ctypes
import re

from conftest import REPO


def declared():
    txt = (REPO / 'include' / 'sawsim_b200.h').read_text()
    return sorted(set(re.findall(r'\b(ss_[a-z0-9_]+)\s*\(', txt)))


def test_header_and_binding_agree():
    from sawsim_b200 import _lib
    assert declared() == sorted(n for n, _, _ in _lib.SIGNATURES)


def test_library_exports_all(built_lib):
    lib = ctypes.CDLL(str(built_lib))
    for name in declared():
        assert hasattr(lib, name), name


def test_python_binding_loads(built_lib):
    from sawsim_b200 import _lib
    lib = _lib.load()
    assert lib.ss_last_error(None) == b'null handle'


def _prototypes():
    """(return type, name, [parameter types]) of every declaration in the header."""
    txt = (REPO / 'include' / 'sawsim_b200.h').read_text()
    txt = re.sub(r'/\*.*?\*/', ' ', txt, flags=re.S)
    out = []
    for ret, name, params in re.findall(r'(?m)^((?:const\s+)?[a-z_0-9]+\s*\**)\s*(ss_[a-z0-9_]+)\s*\(([^)]*)\)\s*;',
                                        txt):
        types = []
        for p in params.split(','):
            p = ' '.join(p.split())
            # drop the parameter name: the last identifier, keeping the stars with the type
            m = re.match(r'^(.*?[\s*])([A-Za-z_][A-Za-z_0-9]*)$', p)
            types.append(m.group(1).replace(' ', '') if m else p.replace(' ', ''))
        out.append((ret.replace(' ', ''), name, types))
    return out


def _compatible(ctype, ct):
    """Is ctypes type ``ct`` a faithful binding of the C parameter type ``ctype``?"""
    C = ctypes
    scalars = {'int': C.c_int, 'int64_t': C.c_int64, 'double': C.c_double}
    if ctype in scalars:
        return ct is scalars[ctype]
    if ctype in ('constchar*',):
        return ct is C.c_char_p
    if ctype in ('ss_handle*', 'constss_handle*', 'void*'):
        return ct is C.c_void_p
    if ctype == 'ss_handle**':
        return ct is C.POINTER(C.c_void_p)
    pointee = {'double*': C.c_double, 'constdouble*': C.c_double, 'int64_t*': C.c_int64,
               'constint64_t*': C.c_int64, 'int32_t*': C.c_int32, 'constint32_t*': C.c_int32, 'int*': C.c_int}
    if ctype in pointee:
        # typed pointer of the same element type, or an untyped device address
        return ct is C.c_void_p or ct is C.POINTER(pointee[ctype])
    raise AssertionError(f'unmapped C type {ctype!r}')


def test_binding_types_match_header():
    """Every ctypes row has the header's parameter count and compatible types, so
    that no argument is passed with the wrong width."""
    from sawsim_b200 import _lib
    rows = {n: (r, a) for n, r, a in _lib.SIGNATURES}
    protos = _prototypes()
    assert sorted(n for _, n, _ in protos) == declared()
    rets = {'int': ctypes.c_int, 'void': None, 'constchar*': ctypes.c_char_p}
    for ret, name, params in protos:
        res, args = rows[name]
        assert res is rets[ret], name
        assert len(args) == len(params), (name, len(args), len(params))
        for i, (p, a) in enumerate(zip(params, args)):
            assert _compatible(p, a), (name, i, p, a)
