"""``nef_class``: frozen attrs classes with the reference's helper methods.

Mirrors nefct/base/base.py:29-177 (NefBaseClass / nef_class): every
annotated field becomes an optional attrs attribute (default None unless the
class gives one), instances are frozen, and ``update`` / ``asdict`` /
``keys`` / ``values`` / ``items`` behave as in the reference.
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
