"""The C ABI's struct layouts, checked field by field against the compiled
library's own table (tk_abi_layout): the ctypes and numpy mirrors the tests and
bench use, and the Rust #[repr(C)] declarations of the FFI crate in
INTEGRATION.md. The reference checks its record layouts the same way
(src/shared/gpu_coarse.rs:210-286, src/shared/draw_record.rs:165-175)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from tileink_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]

CTYPES_MIRRORS = {
    "tk_scene_desc": N.SceneDesc, "tk_image_desc": N.ImageDesc, "tk_stats": N.Stats,
    "tk_gradient_stop": N.GradientStop, "tk_brush_desc": N.BrushDesc, "tk_sdf_shape": N.SdfShape,
    "tk_flatten_desc": N.FlattenDesc, "tk_diff_scene": N.DiffScene, "tk_batch_info": N.BatchInfo,
    "tk_tune_result": N.TuneResult, "tk_gen_params": N.GenParams, "tk_damage": N.Damage,
    "tk_incremental_stats": N.IncrementalStats, "tk_abi_field": N.AbiField,
}
DTYPE_MIRRORS = {
    "tk_line": N.LINE_DTYPE, "tk_affine": N.AFFINE_DTYPE, "tk_path_record": N.PATH_DTYPE,
    "tk_pixel_bounds": N.BOUNDS_DTYPE, "tk_draw_record": N.DRAW_DTYPE, "tk_layer_record": N.LAYER_DTYPE,
    "tk_ptcl_record": N.PTCL_DTYPE, "tk_line_segment": N.SEGMENT_DTYPE, "tk_segment_range": N.RANGE_DTYPE,
    "tk_tile_record": N.TILE_DTYPE, "tk_op": N.OP_DTYPE, "tk_flatten_el": N.FLATTEN_EL_DTYPE,
    "tk_stroke_polyline": N.POLYLINE_DTYPE, "tk_stroke_desc": N.STROKE_DTYPE,
    "tk_glyph_run": N.GLYPH_RUN_DTYPE, "tk_glyph": N.GLYPH_DTYPE, "tk_glyph_image": N.GLYPH_IMAGE_DTYPE,
    "tk_progressive_blur": N.PROGRESSIVE_DTYPE,
    "tk_filter": N.FILTER_DTYPE,
    "tk_filter_layer": N.FILTER_LAYER_DTYPE,
    "tk_canvas_filter": N.CANVAS_FILTER_DTYPE,
}


@pytest.fixture(scope="module")
def layout():
    return N.abi_layout()


def test_every_header_struct_is_in_the_table(layout):
    names = set()
    for h in ("tileink.h", "tileink_canvas.h", "tileink_diff.h"):
        text = (ROOT / "include" / h).read_text()
        names |= set(re.findall(r"\}\s*(tk_\w+)\s*;", text))
    assert names == set(layout), names ^ set(layout)


def header_fields() -> dict:
    """{struct: [field, ...]} parsed from the three public headers."""
    out = {}
    for h in ("tileink.h", "tileink_canvas.h", "tileink_diff.h"):
        text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / h).read_text(), flags=re.S)
        for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} (\w+);", text, flags=re.S):
            fields = []
            for decl in m.group(2).split(";"):
                decl = decl.strip()
                if not decl:
                    continue
                names = decl.split(None, 2 if decl.startswith("const") else 1)[-1].replace("*", "")
                fields += [re.sub(r"\[.*", "", n).strip() for n in names.split(",")]
            out[m.group(3)] = fields
    return out


def test_table_lists_every_header_field_in_order(layout):
    for name, fields in header_fields().items():
        assert [k for k in layout[name] if k] == fields, name


def test_record_sizes_equal_the_reference_pod_types(layout):
    # src/shared/{line,path,draw_record,line_seg,gpu_coarse}.rs
    want = {"tk_line": 24, "tk_path_record": 76, "tk_draw_record": 124, "tk_layer_record": 12,
            "tk_ptcl_record": 24, "tk_line_segment": 20, "tk_segment_range": 8, "tk_tile_record": 24,
            "tk_affine": 24, "tk_op": 36}
    assert {k: layout[k][""] for k in want} == want


@pytest.mark.parametrize("name", sorted(CTYPES_MIRRORS))
def test_ctypes_mirror_matches_library(layout, name):
    cls = CTYPES_MIRRORS[name]
    lib = layout[name]
    assert C.sizeof(cls) == lib[""]
    fields = [f[0] for f in cls._fields_]
    assert fields == [k for k in lib if k], (fields, list(lib))
    for f in fields:
        d = getattr(cls, f)
        assert (d.offset, d.size) == lib[f], f


@pytest.mark.parametrize("name", sorted(DTYPE_MIRRORS))
def test_numpy_mirror_matches_library(layout, name):
    dt = DTYPE_MIRRORS[name]
    lib = layout[name]
    assert dt.itemsize == lib[""]
    assert list(dt.names) == [k for k in lib if k]
    for f in dt.names:
        sub, off = dt.fields[f][:2]
        assert (off, sub.itemsize) == lib[f], f


# --- the Rust declarations of INTEGRATION.md ----------------------------------

RUST_SCALARS = {"u8": 1, "i8": 1, "u16": 2, "i16": 2, "u32": 4, "i32": 4, "f32": 4, "u64": 8, "i64": 8,
                "f64": 8, "usize": 8, "isize": 8}


def rust_type_layout(ty: str, known: dict) -> tuple[int, int]:
    """(size, align) of a Rust type under #[repr(C)] on a 64-bit target."""
    ty = ty.strip()
    if ty.startswith("*const ") or ty.startswith("*mut ") or ty.startswith("&"):
        return 8, 8
    m = re.fullmatch(r"\[(.+);\s*(\d+)\]", ty)
    if m:
        size, align = rust_type_layout(m.group(1), known)
        return size * int(m.group(2)), align
    if ty in RUST_SCALARS:
        return RUST_SCALARS[ty], RUST_SCALARS[ty]
    if ty in known:
        return known[ty]
    raise AssertionError(f"unknown Rust type {ty}")


def rust_structs(markdown: str) -> dict:
    """Every `pub struct` in the ```rust blocks, with its fields' (offset,
    size) and its size under #[repr(C)]."""
    known: dict = {}
    out: dict = {}
    for block in re.findall(r"```rust\n(.*?)```", markdown, flags=re.S):
        for m in re.finditer(r"pub struct (\w+)\s*\{(.*?)\}", block, flags=re.S):
            body = re.sub(r"//[^\n]*", "", m.group(2))
            fields = re.findall(r"pub\s+(\w+)\s*:\s*([^,]+?)\s*(?:,|$)", body)
            off, align, table = 0, 1, {}
            for name, ty in fields:
                size, a = rust_type_layout(ty, known)
                off = (off + a - 1) // a * a
                table[name] = (off, size)
                off += size
                align = max(align, a)
            size = (off + align - 1) // align * align
            table[""] = size
            known[m.group(1)] = (size, align)
            out[m.group(1)] = table
    return out


def test_integration_rust_declarations_match_library(layout):
    rust = rust_structs((ROOT / "INTEGRATION.md").read_text())
    assert {"tk_op", "tk_image_desc", "tk_scene_desc", "tk_stats"} <= set(rust)
    for name, table in rust.items():
        assert name in layout, name
        lib = layout[name]
        assert table[""] == lib[""], (name, table[""], lib[""])
        assert [k for k in table if k] == [k for k in lib if k], name
        for f in table:
            if f:
                assert table[f] == lib[f], (name, f, table[f], lib[f])


def test_integration_rust_size_asserts_match_library(layout):
    text = (ROOT / "INTEGRATION.md").read_text()
    sizes = {"Line": "tk_line", "PathRecord": "tk_path_record", "DrawRecord": "tk_draw_record",
             "LayerStackRecord": "tk_layer_record", "PtclRecord": "tk_ptcl_record"}
    found = re.findall(r"size_of::<(\w+)>\(\) == (\d+)", text)
    assert len(found) >= 8
    for ty, n in found:
        assert layout[sizes.get(ty, ty)][""] == int(n), ty
    for ty, f, n in re.findall(r"offset_of!\((\w+), (\w+)\) == (\d+)", text):
        assert layout[ty][f][0] == int(n), (ty, f)
