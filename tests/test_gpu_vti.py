"""VTI / PVD output through glide_b200.io on the GPU (the pack kernel behind
glide_vti_pack): byte-for-byte the files the reference's own writer produced
from the same inputs (tests/golden/vti/), for 2-D scalars, face-field
vectors, 3-component vectors without the y flip, 3-D layer-major volumes,
and the VTIWriter series with its PVD manifest, synchronous and in the
background.  Larger cases (more arrays than one launch takes, strided views)
are compared with the oracle restatement, which is pinned to the same
files."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden" / "vti"


class FaceField:
    """A field object as the writer sees one: data plus its grid entity."""

    def __init__(self, data, entity):
        self.data = data
        self.grid_entity = entity


@pytest.fixture(scope="module")
def f():
    with np.load(G / "inputs.npz") as z:
        return {k: torch.as_tensor(z[k], device="cuda") for k in z.files}


def test_write_vti_matches_reference_files(f, tmp_path):
    from glide_b200.io import write_vti
    u = FaceField(f["u"], "vertical_facet")
    v = FaceField(f["v"], "horizontal_facet")
    write_vti(tmp_path / "a.vti", {"H": f["H"], "U": [u, v], "B": f["B"]}, 1000.0, origin=(100.0, -50.0),
              time_value=2.5)
    assert (tmp_path / "a.vti").read_bytes() == (G / "scalars_vector2.vti").read_bytes()
    write_vti(tmp_path / "b.vti", {"W": [f["a"], f["b"], f["c"]], "bed": f["bed"]}, 250.0, dy=500.0,
              flip_y=False)
    assert (tmp_path / "b.vti").read_bytes() == (G / "vector3_noflip.vti").read_bytes()
    # E as the enthalpy solver holds it: layer-major storage seen as (ny, nx, nz)
    E_layers = f["E"].permute(2, 0, 1).contiguous()
    E_view = E_layers.permute(1, 2, 0)
    assert not E_view.is_contiguous()
    write_vti(tmp_path / "c.vti", {"E": E_view, "T": f["T"]}, 2000.0, dz=0.5, origin=(1.0, 2.0, 3.0),
              time_value=10)
    assert (tmp_path / "c.vti").read_bytes() == (G / "volume.vti").read_bytes()


@pytest.mark.parametrize("background", [False, True])
def test_vti_writer_series_matches_reference_files(f, tmp_path, background):
    from glide_b200.io import VTIWriter
    H = FaceField(f["H"].clone(), "cell")
    u = FaceField(f["u"], "vertical_facet")
    v = FaceField(f["v"], "horizontal_facet")
    w = VTIWriter(out_dir=tmp_path, base="dome", dx=1000.0, origin=(0.0, 0.0), background=background,
                  static_fields={"bed": f["bed"]},
                  dynamic_fields={"H": H, "U": [u, v], "Hsq": lambda: H.data * 2.0})
    w.initialize(None)
    w.append(None, time=0.0)
    H.data.copy_(f["H1"])  # the next step overwrites the field in place
    w.append(None, time=5.0)
    w.write_pvd()
    for name in ("dome_static.vti", "dome_0000.vti", "dome_0001.vti", "dome.pvd"):
        assert (tmp_path / name).read_bytes() == (G / "series" / name).read_bytes(), name


def test_many_arrays_and_pitched_views_match_oracle(tmp_path):
    """20 arrays (two pack launches), views into pitched storage, binary32
    and binary64, a larger 3-D volume."""
    from glide_b200.io import write_vti
    from oracle import vti_oracle as vo
    rng = np.random.default_rng(7)
    ny, nx = 37, 53
    data_t, data_np = {}, {}
    for q in range(20):
        big = rng.normal(size=(ny, nx + 11)).astype(np.float32 if q % 2 else np.float64)
        data_t[f"f{q}"] = torch.as_tensor(big, device="cuda")[:, 3:3 + nx]
        data_np[f"f{q}"] = big[:, 3:3 + nx]
    ufaces = rng.normal(size=(ny, nx + 1))
    data_t["U"] = [FaceField(torch.as_tensor(ufaces, device="cuda"), "vertical_facet"),
                   torch.as_tensor(data_np["f1"], device="cuda")]
    data_np["U"] = [vo.to_cell(ufaces, "vertical_facet"), data_np["f1"]]
    write_vti(tmp_path / "m.vti", data_t, 90.0, origin=(-5.0, 7.5), time_value=1.25)
    assert (tmp_path / "m.vti").read_bytes() == vo.vti_bytes(data_np, 90.0, origin=(-5.0, 7.5), time_value=1.25)
    nz = 9
    vol = rng.normal(size=(nz, ny, nx))
    write_vti(tmp_path / "v.vti", {"E": torch.as_tensor(vol, device="cuda").permute(1, 2, 0)}, 90.0, dz=0.125,
              flip_y=False)
    assert (tmp_path / "v.vti").read_bytes() == vo.vti_bytes({"E": vol.transpose(1, 2, 0)}, 90.0, dz=0.125,
                                                              flip_y=False)


def test_write_vti_argument_errors(f, tmp_path):
    from glide_b200.io import write_vti
    with pytest.raises(ValueError, match="dz must be provided"):
        write_vti(tmp_path / "x.vti", {"E": f["E"]}, 1.0)
    with pytest.raises(NotImplementedError):
        write_vti(tmp_path / "x.vti", {"E": f["E"], "U": [f["a"], f["c"]]}, 1.0, dz=1.0)
    with pytest.raises(ValueError, match="expected 2D"):
        write_vti(tmp_path / "x.vti", {"H": f["H"], "E": f["E"]}, 1.0)
    with pytest.raises(ValueError, match="2D or 3D"):
        write_vti(tmp_path / "x.vti", {"s": torch.zeros(4, device="cuda")}, 1.0)
    with pytest.raises(ValueError):
        write_vti(tmp_path / "x.vti", {"H": f["H"], "K": torch.zeros(3, 3, device="cuda")}, 1.0)
