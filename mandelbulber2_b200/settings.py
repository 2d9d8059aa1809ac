"""mandelbulber2 settings files (.fract) read through the C-ABI.

`load_from_string` and `load_from_file` mirror cSettings::LoadFromString and
cSettings::LoadFromFile (src/settings.cpp:475-527) for the parameters the DE
path reads; `mbr_fract_parse` (fract_loader.cpp) does the reading.  The
result carries the status: MBR_OK when the scene's geometry is fully
representable, MBR_EUNSUPPORTED (structs filled, report naming what is not
built), MBR_EINVAL (not a settings file or a malformed value).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import abi

REPORT_SIZE = 1 << 16


@dataclass
class Settings:
    status: int
    scene: abi.Scene
    camera: abi.Camera
    params: abi.RenderParams
    report: str

    @property
    def ok(self) -> bool:
        return self.status == abi.MBR_OK

    def unsupported(self) -> list[str]:
        return [ln[len("unsupported: "):] for ln in self.report.splitlines() if ln.startswith("unsupported: ")]


def load_from_string(text: str | bytes) -> Settings:
    lib = abi.load()
    data = text.encode("utf-8", "replace") if isinstance(text, str) else bytes(text)
    sc, cam, p = abi.Scene(), abi.Camera(), abi.RenderParams()
    rep = C.create_string_buffer(REPORT_SIZE)
    st = lib.mbr_fract_parse(data, C.byref(sc), C.byref(cam), C.byref(p), rep, REPORT_SIZE)
    return Settings(int(st), sc, cam, p, rep.value.decode("utf-8", "replace"))


def load_from_file(path: str) -> Settings:
    with open(path, "rb") as f:
        return load_from_string(f.read())
