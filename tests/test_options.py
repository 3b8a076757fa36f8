"""Option files (the reference console's OptionManager, FasterStereoConsole/option_manager.cpp):
read, written and classified like the reference (CPU only)."""
import fasterstereocuda_b200 as fsc
from fasterstereocuda_b200.options import OptionManager, _atof, _atoi

OPTION1 = """<?xml version="1.0" encoding="UTF-8" standalone="no"?>
<Option1>
    <View>
        <width>640</width>
        <height>360</height>
    </View>
    <Stereo>
        <disp_min>-8</disp_min>
        <disp_max>120</disp_max>
        <layers_num>2</layers_num>
        <do_consistency_check>0</do_consistency_check>
        <do_remove_peaks>1</do_remove_peaks>
        <do_smooth>1</do_smooth>
    </Stereo>
</Option1>
"""


def test_c_number_parsing():
    assert _atoi("  12abc") == 12 and _atoi("abc") == 0 and _atoi("-7") == -7 and _atoi("+3") == 3
    assert _atoi("4294967297") == 1  # the int32 field keeps the low 32 bits
    assert _atof(" 3.5e2x") == 350.0 and _atof("-.25") == -0.25 and _atof("x1") == 0.0 and _atof("7") == 7.0


def test_load_option1(tmp_path):
    p = tmp_path / "option.xml"
    p.write_text(OPTION1)
    m = OptionManager()
    assert m.GaussType(str(p)) == OptionManager.OPTION_1
    o = fsc.StereoOption1()
    assert m.Load(str(p), o)
    assert (o.width, o.height, o.min_disp, o.max_disp, o.num_layers) == (640, 360, -8, 120, 2)
    assert (o.do_lr_check, o.do_rm_peaks, o.do_smooth) == (False, True, True)


def test_missing_file_is_written_from_the_option_and_reads_back(tmp_path):
    m = OptionManager()
    p = str(tmp_path / "new.xml")
    o = fsc.StereoOption1(width=1242, height=375, min_disp=0, max_disp=64, num_layers=3, do_smooth=True)
    assert not m.Load(p, o)
    text = open(p).read()
    assert text.startswith('<?xml version="1.0" encoding="UTF-8" standalone="no"?>\n<Option1>')
    assert "<do_smooth>1</do_smooth>" in text and "<disp_max>64</disp_max>" in text
    back = fsc.StereoOption1()
    assert m.Load(p, back)
    assert [getattr(back, f) for f, _ in back._fields_] == [getattr(o, f) for f, _ in o._fields_]


def test_option2_round_trip_with_camera(tmp_path):
    m = OptionManager()
    p = str(tmp_path / "depth.xml")
    epi = fsc.EpipolarStereoParam(x0_left=600.25, y0_left=180.5, x0_right=610.0, y0_right=180.5, baseline=540.0,
                                  focus=720.125)
    o = fsc.StereoOption2(width=1242, height=375, min_depth=5000.0, max_depth=60000.5, num_layers=3, epi=epi)
    assert not m.Load(p, o)
    text = open(p).read()
    assert "<depth_max>60000.500000</depth_max>" in text and "<focus_pix>720.125000</focus_pix>" in text
    assert m.GaussType(p) == OptionManager.OPTION_2
    back = fsc.StereoOption2()
    assert m.Load(p, back)
    assert (back.width, back.height, back.min_depth, back.max_depth, back.num_layers) == (1242, 375, 5000.0, 60000.5, 3)
    assert (back.epi.x0_left, back.epi.y0_left, back.epi.x0_right, back.epi.baseline, back.epi.focus) == \
        (600.25, 180.5, 610.0, 540.0, 720.125)


def test_partial_unparsable_and_foreign_files(tmp_path):
    m = OptionManager()
    # absent elements leave fields unchanged
    p = tmp_path / "partial.xml"
    p.write_text("<Option1><Stereo><disp_max>96</disp_max><layers_num></layers_num></Stereo></Option1>")
    o = fsc.StereoOption1(width=320, height=240, max_disp=64, num_layers=2)
    assert m.Load(str(p), o)
    assert (o.width, o.height, o.max_disp, o.num_layers) == (320, 240, 96, 2)
    # an Option1 file read into StereoOption2 takes the shared fields
    q = tmp_path / "one.xml"
    q.write_text(OPTION1)
    o2 = fsc.StereoOption2(min_depth=1.0)
    assert m.Load(str(q), o2)
    assert (o2.width, o2.num_layers, o2.min_depth, o2.do_lr_check) == (640, 2, 1.0, False)
    # unparsable: rewritten from the option, Load fails, the next Load succeeds
    r = tmp_path / "broken.xml"
    r.write_text("<Option1><View>")
    assert m.GaussType(str(r)) == OptionManager.OPTION_NO
    assert not m.Load(str(r), fsc.StereoOption1(width=99, height=77))
    back = fsc.StereoOption1()
    assert m.Load(str(r), back) and (back.width, back.height) == (99, 77)
    # unknown root, missing file
    s = tmp_path / "other.xml"
    s.write_text("<Settings/>")
    assert m.GaussType(str(s)) == OptionManager.OPTION_NO
    assert m.GaussType(str(tmp_path / "none.xml")) == OptionManager.OPTION_NO
