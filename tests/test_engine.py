"""Scene edit tracking and the render engine's compile sequence (no GPU): a
recording integrator stands in for the device one, and each edit must cause
exactly the calls RenderEngine::startRendering makes in the reference
(src/core/librender/renderengine.cpp:27-114): a compile step runs only when
its edit flag is set, and each one resets the progressive iteration."""
import numpy as np
import pytest

from colvillea_b200 import scenes
from colvillea_b200.engine import RenderEngine, Scene, SceneEditAction as A


class Recorder:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def f(*args, **kw):
            self.calls.append((name, args, kw))
        return f

    def names(self):
        out = [c[0] for c in self.calls]
        self.calls.clear()
        return out


def small_scene():
    return Scene.fromScene(scenes.config1(seed=3, width=32, height=32))


def test_flag_values():
    # scene.h:27-69
    assert A.ShapeEdited == 1 and A.ShapeAdded == 2 and A.ShapeRemoved == 4
    assert A.MaterialEdited == 8 and A.EntityEdited == 64 and A.EmitterEdited == 512 and A.TexturesEdited == 4096
    assert A.AnyShapeModification == 7 and A.AnyEmitterModification == (7 << 9)


def test_initial_compile_sequence():
    s, it = small_scene(), Recorder()
    assert s.hasAction(A.ShapeAdded | A.MaterialAdded | A.EntityAdded | A.EmitterAdded)
    eng = RenderEngine(it, s)
    eng.startRendering(4)
    assert it.names() == ["buildMaterials", "resetIterationIndex", "buildBLAS", "buildTLAS", "resetIterationIndex",
                          "buildEmitters", "resetIterationIndex", "updateCamera", "render"]
    assert s.actions == A.NONE
    # no edits: progressive accumulation continues (camera unchanged is a no-op in the integrator)
    eng.startRendering(1)
    assert it.names() == ["updateCamera", "render"]
    # a textured scene uploads its textures with the materials
    ts, tit = Scene.fromScene(scenes.textured(0, 32, 32)), Recorder()
    RenderEngine(tit, ts).startRendering(1)
    calls = list(tit.calls)
    assert [c[0] for c in calls[:3]] == ["buildTextures", "buildMaterials", "resetIterationIndex"]
    assert len(calls[0][1][0]) == 7 and calls[1][1][0][0].reflectance_texture == 1


def test_vertex_edit_refits():
    s, it = small_scene(), Recorder()
    eng = RenderEngine(it, s, bvh_update="refit")
    eng.startRendering()
    it.names()
    m = s.meshes[5]
    p = m.positions + np.float32([0.0, 0.25, 0.0])
    m.updateVertices(p)
    assert s.actions == A.ShapeEdited
    eng.startRendering()
    calls = list(it.calls)
    assert [c[0] for c in calls] == ["updateVertices", "updateCamera", "render"]
    name, args, kw = calls[0]
    assert args[0] == 5 and np.array_equal(args[1], p) and kw == {"bvh": "refit"}
    it.names()
    # two meshes edited: two updates, in mesh order
    s.meshes[7].updateVertices(s.meshes[7].positions * 1.01)
    s.meshes[2].updateVertices(s.meshes[2].positions * 0.99)
    eng.startRendering()
    assert [(c[0], c[1][0] if c[0] == "updateVertices" else None) for c in it.calls[:2]] == \
        [("updateVertices", 2), ("updateVertices", 7)]


def test_material_and_emitter_edits():
    s, it = small_scene(), Recorder()
    eng = RenderEngine(it, s)
    eng.startRendering()
    it.names()
    s.materials[1].set(reflectance=(0.9, 0.1, 0.1))
    eng.startRendering()
    assert it.names() == ["buildMaterials", "resetIterationIndex", "updateCamera", "render"]
    s.emitters[0].set(intensity=(5.0, 5.0, 5.0))
    eng.startRendering()
    assert it.names() == ["buildEmitters", "resetIterationIndex", "updateCamera", "render"]
    with pytest.raises(AttributeError):
        s.materials[0].set(colour=1)


def test_entity_edits_rebuild():
    s, it = small_scene(), Recorder()
    eng = RenderEngine(it, s)
    eng.startRendering()
    it.names()
    e = s.entities[3]
    e.setTransform((1, 0, 0, 0.5, 0, 1, 0, 0, 0, 0, 1, 0))
    # a vertex edit in the same frame is covered by the full rebuild
    s.meshes[4].updateVertices(s.meshes[4].positions)
    eng.startRendering()
    names = it.names()
    assert names == ["buildBLAS", "buildTLAS", "resetIterationIndex", "updateCamera", "render"]
    # removing the only entity of a mesh removes the mesh: ids shift
    n_meshes = len(s.meshes)
    s.removeEntity(s.entities[2])
    assert s.hasAction(A.EntityRemoved | A.ShapeRemoved) and len(s.meshes) == n_meshes - 1
    eng.startRendering()
    blas, tlas = it.calls[0], it.calls[1]
    assert blas[0] == "buildBLAS" and len(blas[1][0]) == n_meshes - 1
    inst = tlas[1][0]
    assert len(inst) == len(s.entities) and max(i[0] for i in inst) == n_meshes - 2
    it.names()
    with pytest.raises(ValueError):
        s.removeMaterial(s.entities[0].material)


def test_update_vertices_checks():
    s = small_scene()
    m = s.meshes[1]
    with pytest.raises(ValueError):
        m.updateVertices(m.positions[:-1])
    bad = m.positions.copy()
    bad[0, 0] = np.nan
    with pytest.raises(ValueError):
        m.updateVertices(bad)
    assert not s.hasAction(A.ShapeEdited) or s.hasAction(A.ShapeAdded)


def test_texture_edits():
    s, it = Scene.fromScene(scenes.textured(0, 32, 32)), Recorder()
    eng = RenderEngine(it, s)
    eng.startRendering()
    it.names()
    t = s.textures[2]
    t.setTexels(t.desc.texels * 0.5)
    assert s.actions == A.TexturesEdited
    eng.startRendering()
    assert it.names() == ["buildTextures", "buildMaterials", "resetIterationIndex", "updateCamera", "render"]
    # a new texture on a material; indices follow the scene's texture order
    nt = s.createTexture(scenes.roughness_texture(16, np.random.default_rng(0)))
    s.materials[3].set(roughness_texture=nt)
    eng.startRendering()
    mats = it.calls[1][1][0]
    assert mats[3].roughness_texture == len(s.textures)
    it.names()
    with pytest.raises(ValueError):
        s.removeTexture(nt)
    s.materials[3].set(roughness_texture=None)
    s.removeTexture(nt)
    eng.startRendering()
    assert it.calls[1][1][0][3].roughness_texture == 0
