"""Option files of the reference's console (FasterStereoConsole/option_manager.h, option_manager.cpp).

An option file is XML with root <Option1> (search range as disparities, read into StereoOption1)
or <Option2> (search range as depths plus the rectified camera, read into StereoOption2):

    <Option1>                          <Option2>
      <View> width height </View>        <View> width height </View>
      <Stereo> disp_min disp_max         <Stereo> depth_min depth_max layers_num
               layers_num                         do_consistency_check do_remove_peaks do_smooth
               do_consistency_check      </Stereo>
               do_remove_peaks           <Camera> x0_left_pix y0_left_pix x0_right_pix y0_right_pix
               do_smooth </Stereo>                baseline_mm focus_pix </Camera>
    </Option1>                         </Option2>

Behaviour follows the reference's OptionManager: a missing or unparsable file is written with the
option's current values and Load returns False; elements that are absent leave their fields
unchanged; integers are read like C atoi and reals like C atof (leading number, 0 when there is
none). An element present without text is skipped here (the reference passes a null pointer to
atoi there).
"""
from __future__ import annotations

import os
import re
import xml.etree.ElementTree as ET

from . import StereoOption1, StereoOption2

_INT = re.compile(r"\s*([+-]?\d+)")
_REAL = re.compile(r"\s*([+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))", re.IGNORECASE)


def _atoi(text: str) -> int:
    m = _INT.match(text)
    if not m:
        return 0
    v = int(m.group(1))
    return (v + 2**31) % 2**32 - 2**31  # the int32 field keeps the low 32 bits


def _atof(text: str) -> float:
    m = _REAL.match(text)
    return float(m.group(1)) if m else 0.0


def _cxx_to_string(v) -> str:
    """std::to_string of the value's C++ type: integers and bools in decimal, reals as %f."""
    if isinstance(v, bool):
        return str(int(v))
    if isinstance(v, int):
        return str(v)
    return "%f" % v


class OptionManager:
    """OptionManager (FasterStereoConsole/option_manager.h:17-56)."""

    OPTION_1, OPTION_2, OPTION_NO = 0, 1, 2

    def GaussType(self, path: str) -> int:
        """OptionManager::GaussType (option_manager.cpp:18-44): the kind of option file at `path`."""
        root = self._root(path)
        if root is None:
            return self.OPTION_NO
        return {"Option1": self.OPTION_1, "Option2": self.OPTION_2}.get(root.tag, self.OPTION_NO)

    def Load(self, path: str, opt) -> bool:
        """OptionManager::Load (option_manager.cpp:46-111 for StereoOption1, 113-208 for
        StereoOption2): fields of `opt` from the file; False (and the file written from `opt`) when
        the file is missing or unparsable."""
        if not isinstance(opt, (StereoOption1, StereoOption2)):
            raise TypeError("opt must be a StereoOption1 or a StereoOption2")
        if not os.path.exists(path):
            self._save(path, opt)
            return False
        root = self._root(path)
        if root is None:
            if self._save(path, opt):
                print(f"option file was created in {path}")
            return False
        self._read(root.find("View"), opt, {"width": ("width", _atoi), "height": ("height", _atoi)})

        def flag(t):
            return bool(_atoi(t))
        stereo = {"layers_num": ("num_layers", _atoi), "do_consistency_check": ("do_lr_check", flag),
                  "do_remove_peaks": ("do_rm_peaks", flag), "do_smooth": ("do_smooth", flag)}
        if isinstance(opt, StereoOption1):
            stereo.update({"disp_min": ("min_disp", _atoi), "disp_max": ("max_disp", _atoi)})
            self._read(root.find("Stereo"), opt, stereo)
        else:
            stereo.update({"depth_min": ("min_depth", _atof), "depth_max": ("max_depth", _atof)})
            self._read(root.find("Stereo"), opt, stereo)
            cam = {"x0_left_pix": "x0_left", "y0_left_pix": "y0_left", "x0_right_pix": "x0_right",
                   "y0_right_pix": "y0_right", "baseline_mm": "baseline", "focus_pix": "focus"}
            self._read(root.find("Camera"), opt.epi, {k: (f, _atof) for k, f in cam.items()})
        return True

    # -------------------------------------------------------------------------------------------
    @staticmethod
    def _root(path: str):
        if not os.path.exists(path):
            return None
        try:
            return ET.parse(path).getroot()
        except ET.ParseError:
            return None

    @staticmethod
    def _read(section, target, keys) -> None:
        if section is None:
            return
        for tag, (field, conv) in keys.items():
            el = section.find(tag)
            if el is not None and el.text is not None:
                setattr(target, field, conv(el.text))

    @staticmethod
    def _save(path: str, opt) -> bool:
        """OptionManager::Save (option_manager.cpp:210-342): the option as an option file."""
        one = isinstance(opt, StereoOption1)
        root = ET.Element("Option1" if one else "Option2")
        view = ET.SubElement(root, "View")
        stereo = ET.SubElement(root, "Stereo")
        fields = [(view, "width", int(opt.width)), (view, "height", int(opt.height))]
        if one:
            fields += [(stereo, "disp_min", int(opt.min_disp)), (stereo, "disp_max", int(opt.max_disp))]
        else:
            fields += [(stereo, "depth_min", float(opt.min_depth)), (stereo, "depth_max", float(opt.max_depth))]
        fields += [(stereo, "layers_num", int(opt.num_layers)), (stereo, "do_consistency_check", bool(opt.do_lr_check)),
                   (stereo, "do_remove_peaks", bool(opt.do_rm_peaks)), (stereo, "do_smooth", bool(opt.do_smooth))]
        if not one:
            cam = ET.SubElement(root, "Camera")
            e = opt.epi
            fields += [(cam, "x0_left_pix", float(e.x0_left)), (cam, "y0_left_pix", float(e.y0_left)),
                       (cam, "x0_right_pix", float(e.x0_right)), (cam, "y0_right_pix", float(e.y0_right)),
                       (cam, "baseline_mm", float(e.baseline)), (cam, "focus_pix", float(e.focus))]
        for parent, tag, value in fields:
            ET.SubElement(parent, tag).text = _cxx_to_string(value)
        ET.indent(root, space="    ")
        text = '<?xml version="1.0" encoding="UTF-8" standalone="no"?>\n' + ET.tostring(root, encoding="unicode")
        try:
            with open(path, "w", encoding="utf-8") as f:
                f.write(text + "\n")
        except OSError:
            print("save option files failed!")
            return False
        return True
