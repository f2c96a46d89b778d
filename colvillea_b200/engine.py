"""Scene editing and the render engine's compile step: the reference's
dirty-flag model over the integrator API.

* `SceneEditAction` has the reference's flag values
  (include/colvillea/librender/scene.h:25-92).
* `Scene` holds meshes, materials, entities (mesh + material + transform),
  emitters and the camera.  Its create/remove calls and the nodes' setters
  record edit actions, as the reference's Scene::add* and node setters do
  (scene.h:218-330).  `TriangleMesh.updateVertices` is the reference's
  commented-out shape edit (include/colvillea/nodes/shapes/trianglemesh.h:
  111-118), and it marks ShapeEdited.
* `RenderEngine.startRendering` runs the compile sequence of
  RenderEngine::startRendering (src/core/librender/renderengine.cpp:27-114):
  materials, entities, acceleration structures, emitters, then the camera.
  Each compile that runs resets the progressive iteration, then the edit
  actions are cleared and the integrator renders.

The one difference from the reference is the ShapeEdited path.  Vertex edits
that add or remove no shape and change no entity go through
`Integrator.updateVertices`, which refits the BVH on the device (or
rebuilds it, by `bvh_update`).  Any added or removed shape or entity rebuilds
meshes and instances, as the reference's buildBLAS/buildTLAS do
(scene.cpp:186-243).
"""
import enum

import numpy as np

from . import scenes


class SceneEditAction(enum.IntFlag):
    """EditActionType (scene.h:27-69)."""
    NONE = 0
    ShapeEdited = 1
    ShapeAdded = 1 << 1
    ShapeRemoved = 1 << 2
    MaterialEdited = 1 << 3
    MaterialAdded = 1 << 4
    MaterialRemoved = 1 << 5
    EntityEdited = 1 << 6
    EntityAdded = 1 << 7
    EntityRemoved = 1 << 8
    EmitterEdited = 1 << 9
    EmitterAdded = 1 << 10
    EmitterRemoved = 1 << 11
    TexturesEdited = 1 << 12
    TexturesAdded = 1 << 13
    TexturesRemoved = 1 << 14
    AnyShapeModification = ShapeEdited | ShapeAdded | ShapeRemoved
    AnyMaterialModification = MaterialEdited | MaterialAdded | MaterialRemoved
    AnyEntityModification = EntityEdited | EntityAdded | EntityRemoved
    AnyEmitterModification = EmitterEdited | EmitterAdded | EmitterRemoved
    AnyTextureModification = TexturesEdited | TexturesAdded | TexturesRemoved


A = SceneEditAction


class _Node:
    def __init__(self, scene):
        self._scene = scene


class TriangleMesh(_Node):
    """Vertex arrays as float32 (n, 3) / (n, 2), triangles as uint32 (t, 3)."""

    def __init__(self, scene, positions, normals, tangents, uvs, indices):
        super().__init__(scene)
        self.positions = np.ascontiguousarray(positions, np.float32)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32)
        self.tangents = np.ascontiguousarray(tangents, np.float32)
        self.uvs = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
        self.indices = np.ascontiguousarray(indices, np.uint32)

    def as_mesh(self):
        return scenes.Mesh(self.positions, self.normals, self.tangents, self.uvs, self.indices)

    def updateVertices(self, positions, normals=None, tangents=None):
        """New positions (same count, same triangles); normals/tangents None: kept."""
        p = np.ascontiguousarray(positions, np.float32)
        if p.shape != self.positions.shape:
            raise ValueError(f"positions must have shape {self.positions.shape}, got {p.shape}")
        if not np.all(np.isfinite(p)):
            raise ValueError("positions must be finite")
        self.positions = p
        if normals is not None:
            self.normals = np.ascontiguousarray(normals, np.float32).reshape(p.shape)
        if tangents is not None:
            self.tangents = np.ascontiguousarray(tangents, np.float32).reshape(p.shape)
        self._scene._edited_meshes.add(id(self))
        self._scene._edit(A.ShapeEdited)


class Texture(_Node):
    """An image texture (ImageTexture2D, src/core/nodes/textures/imagetex2d.cpp)."""

    def __init__(self, scene, desc):
        super().__init__(scene)
        self.desc = desc

    def setTexels(self, texels, srgb=None):
        self.desc.texels = texels
        if srgb is not None:
            self.desc.srgb = srgb
        self._scene._edit(A.TexturesEdited)


TEXTURE_SLOTS = ("reflectance_texture", "roughness_texture", "normal_texture")


class Material(_Node):
    """A scenes.Material whose setters mark MaterialEdited.  Its texture slots
    hold Texture nodes (or None); compiling turns them into the 1-based
    indices the integrator takes."""

    def __init__(self, scene, desc, textures=None):
        super().__init__(scene)
        self.desc = desc
        self.textures = {k: None for k in TEXTURE_SLOTS}
        self.textures.update(textures or {})

    def set(self, **fields):
        for k, v in fields.items():
            if k in TEXTURE_SLOTS:
                if v is not None and v not in self._scene.textures:
                    raise ValueError("texture is not in the scene")
                self.textures[k] = v
            elif not hasattr(self.desc, k):
                raise AttributeError(k)
            else:
                setattr(self.desc, k, v)
        self._scene._edit(A.MaterialEdited)

    def setNormalmap(self, texture):
        """Material::setNormalmap (libkernel/base/material.h:91)."""
        self.set(normal_texture=texture)

    def compile(self, tex_index):
        d = scenes.Material(**vars(self.desc))
        for k in TEXTURE_SLOTS:
            t = self.textures[k]
            setattr(d, k, 0 if t is None else tex_index[id(t)] + 1)
        return d


class Emitter(_Node):
    """A scenes.Emitter whose setters mark EmitterEdited."""

    def __init__(self, scene, desc):
        super().__init__(scene)
        self.desc = desc

    def set(self, **fields):
        for k, v in fields.items():
            if not hasattr(self.desc, k):
                raise AttributeError(k)
            setattr(self.desc, k, v)
        self._scene._edit(A.EmitterEdited)


class Entity(_Node):
    """Shape + material + 3x4 row-major transform (librender/entity.h)."""

    def __init__(self, scene, mesh, material, transform):
        super().__init__(scene)
        self.mesh, self.material = mesh, material
        self.transform = tuple(float(x) for x in transform)

    def setTransform(self, transform):
        self.transform = tuple(float(x) for x in transform)
        self._scene._edit(A.EntityEdited)

    def setMaterial(self, material):
        self.material = material
        self._scene._edit(A.EntityEdited)


class Scene:
    """Scene API (scene.h:106-400) with edit tracking."""

    def __init__(self):
        self.meshes, self.materials, self.entities, self.emitters, self.textures = [], [], [], [], []
        self.camera = None
        self.width = self.height = None
        self.actions = A.NONE
        self._edited_meshes = set()
        self._camera_dirty = False

    @staticmethod
    def createScene():
        return Scene()

    def _edit(self, action):
        self.actions |= action

    def hasAction(self, action):
        return bool(self.actions & action)

    # --- creation (Scene::create*, add*) --------------------------------------
    def createTriangleMesh(self, positions, normals, tangents, uvs, indices):
        m = TriangleMesh(self, positions, normals, tangents, uvs, indices)
        self.meshes.append(m)
        self._edit(A.ShapeAdded)
        return m

    def createTexture(self, desc):
        """Scene::createTexture (scene.cpp:78-94) from a scenes.Texture."""
        t = Texture(self, desc)
        self.textures.append(t)
        self._edit(A.TexturesAdded)
        return t

    def createMaterial(self, desc, **textures):
        """A material from a scenes.Material (its texture indices ignored) and
        Texture nodes for the slots given (reflectance_texture=..., ...)."""
        for k, t in textures.items():
            if k not in TEXTURE_SLOTS or (t is not None and t not in self.textures):
                raise ValueError(f"bad texture slot {k}")
        m = Material(self, desc, textures)
        self.materials.append(m)
        self._edit(A.MaterialAdded)
        return m

    def createEntity(self, mesh, material, transform=scenes.IDENTITY):
        if mesh not in self.meshes or material not in self.materials:
            raise ValueError("entity refers to a mesh or material that is not in the scene")
        e = Entity(self, mesh, material, transform)
        self.entities.append(e)
        self._edit(A.EntityAdded)
        return e

    def createEmitter(self, desc):
        e = Emitter(self, desc)
        self.emitters.append(e)
        self._edit(A.EmitterAdded)
        return e

    def setCamera(self, camera12):
        self.camera = np.ascontiguousarray(camera12, np.float32).reshape(12)

    # --- removal --------------------------------------------------------------
    def removeEntity(self, entity):
        self.entities.remove(entity)
        self._edit(A.EntityRemoved)
        if not any(e.mesh is entity.mesh for e in self.entities):
            self.meshes.remove(entity.mesh)
            self._edited_meshes.discard(id(entity.mesh))
            self._edit(A.ShapeRemoved)

    def removeMaterial(self, material):
        if any(e.material is material for e in self.entities):
            raise ValueError("material is used by an entity")
        self.materials.remove(material)
        self._edit(A.MaterialRemoved)

    def removeTexture(self, texture):
        if any(t is texture for m in self.materials for t in m.textures.values()):
            raise ValueError("texture is used by a material")
        self.textures.remove(texture)
        self._edit(A.TexturesRemoved)

    def removeEmitter(self, emitter):
        self.emitters.remove(emitter)
        self._edit(A.EmitterRemoved)

    # --- compilation (Scene::compile*, collect*) ------------------------------
    def compileTextures(self):
        if self.hasAction(A.AnyTextureModification):
            return [t.desc for t in self.textures]
        return None

    def compileMaterials(self):
        """Materials with texture indices; also after texture edits, since
        indices move when textures are added or removed."""
        if self.hasAction(A.AnyMaterialModification | A.AnyTextureModification):
            idx = {id(t): i for i, t in enumerate(self.textures)}
            return [m.compile(idx) for m in self.materials]
        return None

    def needsInstanceBuild(self):
        """Shapes or entities added, removed or edited: meshes and instances are
        rebuilt (buildBLAS + buildTLAS + buildGeometryEntities)."""
        return self.hasAction(A.ShapeAdded | A.ShapeRemoved | A.AnyEntityModification)

    def collectMeshes(self):
        return [m.as_mesh() for m in self.meshes]

    def collectInstances(self):
        mid = {id(m): i for i, m in enumerate(self.meshes)}
        mat = {id(m): i for i, m in enumerate(self.materials)}
        return [(mid[id(e.mesh)], mat[id(e.material)], e.transform) for e in self.entities]

    def collectEditedMeshes(self):
        """(mesh index, mesh) of the meshes whose vertices changed (ShapeEdited)."""
        if not self.hasAction(A.ShapeEdited):
            return []
        return [(i, m) for i, m in enumerate(self.meshes) if id(m) in self._edited_meshes]

    def compileEmitters(self):
        if self.hasAction(A.AnyEmitterModification):
            return [e.desc for e in self.emitters]
        return None

    def resetSceneEditActions(self):
        self.actions = A.NONE
        self._edited_meshes.clear()

    @staticmethod
    def fromScene(desc):
        """An editable Scene holding a scenes.Scene's meshes, materials,
        instances, emitters and camera (all marked added)."""
        s = Scene()
        ms = [s.createTriangleMesh(m.positions, m.normals, m.tangents, m.uvs, m.indices) for m in desc.meshes]
        ts = [s.createTexture(scenes.Texture(t.texels, t.srgb)) for t in getattr(desc, "textures", [])]
        mats = [s.createMaterial(scenes.Material(**vars(m)),
                                 **{k: ts[getattr(m, k) - 1] for k in TEXTURE_SLOTS if getattr(m, k, 0)})
                for m in desc.materials]
        for mesh_id, mat, xf in desc.instances:
            s.createEntity(ms[mesh_id], mats[mat], xf)
        for e in desc.emitters:
            s.createEmitter(scenes.Emitter(**vars(e)))
        s.setCamera(desc.camera)
        s.width, s.height = desc.width, desc.height
        return s


class RenderEngine:
    """RenderEngine (src/core/librender/renderengine.cpp:13-123) over an
    Integrator (colvillea_b200.Integrator or anything with its methods)."""

    def __init__(self, integrator, scene, bvh_update="auto"):
        self.integrator, self.scene, self.bvh_update = integrator, scene, bvh_update

    @staticmethod
    def createRenderEngine(integrator, scene, bvh_update="auto"):
        return RenderEngine(integrator, scene, bvh_update)

    def startRendering(self, spp=1):
        self.compileMaterials()
        self.compileEntitiesAndAccelStructs()
        self.compileEmitters()
        if self.scene.camera is None:
            raise RuntimeError("the scene has no camera")
        self.integrator.updateCamera(self.scene.camera)
        self.scene.resetSceneEditActions()
        self.integrator.render(spp)

    def compileMaterials(self):
        """compileMaterials (renderengine.cpp:54-62); textures are uploaded
        with them (the reference uploads at Scene::createTexture)."""
        texs = self.scene.compileTextures()
        mats = self.scene.compileMaterials()
        if texs is not None:
            self.integrator.buildTextures(texs)
        if mats is not None:
            self.integrator.buildMaterials(mats)
            self.integrator.resetIterationIndex()

    def compileEntitiesAndAccelStructs(self):
        """compileEntities + compileAccelStructs (renderengine.cpp:65-101)."""
        sc = self.scene
        if sc.needsInstanceBuild():
            if not sc.entities:
                raise RuntimeError("the scene has no entities")
            self.integrator.buildBLAS(sc.collectMeshes())
            self.integrator.buildTLAS(sc.collectInstances())
            self.integrator.resetIterationIndex()
        else:
            for i, m in sc.collectEditedMeshes():
                self.integrator.updateVertices(i, m.positions, m.normals, m.tangents, bvh=self.bvh_update)

    def compileEmitters(self):
        ems = self.scene.compileEmitters()
        if ems is not None:
            self.integrator.buildEmitters(ems)
            self.integrator.resetIterationIndex()
