"""``nef_class``: frozen attrs classes with the reference's helper methods.

Mirrors nefct/base/base.py:29-177 (NefBaseClass / nef_class): every
annotated field becomes an optional attrs attribute (default None unless the
class gives one), instances are frozen, and ``update`` / ``asdict`` /
``keys`` / ``values`` / ``items`` / ``from_dict`` / ``astype`` behave as in
the reference.
"""
from __future__ import annotations

import attr

__all__ = ["nef_class", "NefBaseClass"]


class NefBaseClass:
    @classmethod
    def keys(cls) -> list:
        return [a.name for a in attr.fields(cls)]

    def values(self) -> list:
        return [getattr(self, k) for k in self.keys()]

    def items(self, recurse: bool = False) -> list:
        return list(attr.asdict(self, recurse=recurse).items())

    def update(self, **kwargs):
        return attr.evolve(self, **kwargs)

    def asdict(self, recurse: bool = False) -> dict:
        return attr.asdict(self, recurse=recurse)

    @classmethod
    def from_dict(cls, dct: dict):
        """Instance from a dict of field values (nefct/base/base.py:98-118):
        missing keys stay None, a nested dict becomes the annotated
        nef_class of its field, numpy booleans become bool."""
        import numpy as np
        if dct is None:
            return cls()
        hints = _field_types(cls)
        kwargs = {}
        for key in cls.keys():
            if key not in dct:
                continue
            val = dct[key]
            type_ = hints.get(key)
            if isinstance(val, dict) and isinstance(type_, type) and issubclass(type_, NefBaseClass):
                val = type_.from_dict(val)
            elif isinstance(val, np.bool_):
                val = bool(val)
            kwargs[key] = val
        return cls(**kwargs)

    def astype(self, cls: type):
        """The same fields as another nef_class (base.py:120-121)."""
        return cls.from_dict(self.asdict(recurse=True))


def _field_types(cls) -> dict:
    """Field annotations resolved to classes (modules here use postponed
    annotations, so they are strings until resolved)."""
    import sys
    import typing
    try:
        return typing.get_type_hints(cls, vars(sys.modules[cls.__module__]))
    except Exception:
        return {}


def nef_class(cls):
    """Decorator: frozen attrs class whose fields all default to None."""
    ann = cls.__dict__.get("__annotations__", {})
    for name in ann:
        if name not in cls.__dict__:
            setattr(cls, name, attr.ib(default=None))
        elif not isinstance(cls.__dict__[name], attr._make._CountingAttr):
            setattr(cls, name, attr.ib(default=cls.__dict__[name]))
    if NefBaseClass in cls.__mro__:
        bases = cls.__bases__
    else:
        bases = tuple(b for b in cls.__bases__ if b is not object) + (NefBaseClass,)
    if bases != cls.__bases__:
        ns = {k: v for k, v in cls.__dict__.items() if k not in ("__dict__", "__weakref__")}
        cls = type(cls.__name__, bases, ns)
    return attr.s(auto_attribs=True, frozen=True, eq=False)(cls)
