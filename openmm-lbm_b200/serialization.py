"""XML serialization of LBMForce in the format of the reference's serialization proxy (LBMForceProxy,
serialization/src/LBMForceProxy.cpp:22-147), written and read as OpenMM's XmlSerializer does: one element per node,
named for the object (the root "Force" for a force), its properties as attributes in the order of their names, the
child nodes in the order in which the proxy creates them, one tab of indentation per level.

The proxy writes version 9 (forceGroup, name, nx, ny, nz, domainsX/Y/Z, particleCopiesCheck, densityHaloExchange,
velocityHaloExchange, density, viscosity, friction, temperature, randomSeed, momentumRemovalFrequency,
machCheckFrequency, couplingScheme, dragScheme, interpolationStencil, fluidFluctuations, wallScheme, machNumberLimit;
children BodyAcceleration, InitialFluidVelocity, Particles, SolidNodes and Faces) and reads versions 1 to 9, where
the settings that an older version lacks keep the values of that time (LBMForceProxy.cpp:75-145).  Integers and
booleans ("1" / "0") are written in decimal, doubles in the shortest form that reads back to the same value.

    xml = XmlSerializer.serialize(force)
    copy = XmlSerializer.deserialize(xml)
"""
import xml.etree.ElementTree as ElementTree
from xml.sax.saxutils import escape

from .force import LBMForce

VERSION = 9


class SerializationError(ValueError):
    """A node that the proxy cannot read (OpenMM's OpenMMException in the reference)."""


class SerializationNode:
    """A node of OpenMM's serialization tree: a name, string properties and child nodes."""

    def __init__(self, name=''):
        self.name = name
        self.properties = {}
        self.children = []

    def createChildNode(self, name):
        child = SerializationNode(name)
        self.children.append(child)
        return child

    def getChildNode(self, name):
        for child in self.children:
            if child.name == name:
                return child
        raise SerializationError("Unknown child '%s' in node '%s'" % (name, self.name))

    def _get(self, name, default, convert):
        if name not in self.properties:
            if default is _REQUIRED:
                raise SerializationError("Unknown property '%s' in node '%s'" % (name, self.name))
            return default
        try:
            return convert(self.properties[name])
        except ValueError:
            raise SerializationError("Property '%s' in node '%s' is not valid: %r" %
                                     (name, self.name, self.properties[name]))

    def setIntProperty(self, name, value):
        self.properties[name] = str(int(value))
        return self

    def getIntProperty(self, name, default=None):
        return self._get(name, _REQUIRED if default is None else default, int)

    def setBoolProperty(self, name, value):
        self.properties[name] = '1' if value else '0'
        return self

    def getBoolProperty(self, name, default=None):
        return self._get(name, _REQUIRED if default is None else default, _parse_bool)

    def setDoubleProperty(self, name, value):
        self.properties[name] = repr(float(value))
        return self

    def getDoubleProperty(self, name, default=None):
        return self._get(name, _REQUIRED if default is None else default, float)

    def setStringProperty(self, name, value):
        self.properties[name] = str(value)
        return self

    def getStringProperty(self, name, default=None):
        return self._get(name, _REQUIRED if default is None else default, str)


_REQUIRED = object()


def _parse_bool(text):
    if text in ('1', 'true'):
        return True
    if text in ('0', 'false'):
        return False
    raise ValueError(text)


def serialize_node(force, node):
    """LBMForceProxy::serialize (LBMForceProxy.cpp:22-71)."""
    node.setIntProperty('version', VERSION)
    node.setIntProperty('forceGroup', force.getForceGroup())
    node.setStringProperty('name', force.getName())
    nx, ny, nz = force.getGridSize()
    node.setIntProperty('nx', nx).setIntProperty('ny', ny).setIntProperty('nz', nz)
    px, py, pz = force.getDomainDecomposition()
    node.setIntProperty('domainsX', px).setIntProperty('domainsY', py).setIntProperty('domainsZ', pz)
    node.setBoolProperty('particleCopiesCheck', force.getParticleCopiesCheck())
    node.setBoolProperty('densityHaloExchange', force.getDensityHaloExchange())
    node.setBoolProperty('velocityHaloExchange', force.getVelocityHaloExchange())
    node.setDoubleProperty('density', force.getFluidDensity())
    node.setDoubleProperty('viscosity', force.getKinematicViscosity())
    node.setDoubleProperty('friction', force.getFriction())
    node.setDoubleProperty('temperature', force.getTemperature())
    node.setIntProperty('randomSeed', force.getRandomNumberSeed())
    node.setIntProperty('momentumRemovalFrequency', force.getFluidMomentumRemovalFrequency())
    node.setIntProperty('machCheckFrequency', force.getMachCheckFrequency())
    node.setIntProperty('couplingScheme', force.getCouplingScheme())
    node.setIntProperty('dragScheme', force.getDragScheme())
    node.setIntProperty('interpolationStencil', force.getInterpolationStencil())
    node.setBoolProperty('fluidFluctuations', force.getFluidFluctuations())
    node.setIntProperty('wallScheme', force.getWallScheme())
    node.setDoubleProperty('machNumberLimit', force.getMachNumberLimit())
    g = force.getBodyAcceleration()
    node.createChildNode('BodyAcceleration').setDoubleProperty('x', g[0]).setDoubleProperty('y', g[1]) \
        .setDoubleProperty('z', g[2])
    u = force.getInitialFluidVelocity()
    node.createChildNode('InitialFluidVelocity').setDoubleProperty('x', u[0]).setDoubleProperty('y', u[1]) \
        .setDoubleProperty('z', u[2])
    particles = node.createChildNode('Particles')
    for i in range(force.getNumParticles()):
        particles.createChildNode('Particle').setIntProperty('index', force.getParticle(i))
    solid = node.createChildNode('SolidNodes')
    for index in force.getSolidNodes():
        solid.createChildNode('Node').setIntProperty('index', index)
    faces = node.createChildNode('Faces')
    for face in range(6):
        v = force.getFaceVelocity(face)
        faces.createChildNode('Face').setIntProperty('type', force.getFaceBoundary(face)) \
            .setDoubleProperty('vx', v[0]).setDoubleProperty('vy', v[1]).setDoubleProperty('vz', v[2]) \
            .setDoubleProperty('density', force.getFaceDensity(face))


def deserialize_node(node):
    """LBMForceProxy::deserialize (LBMForceProxy.cpp:73-147): versions 1 to 9."""
    version = node.getIntProperty('version')
    if version < 1 or version > VERSION:
        raise SerializationError('Unsupported version number')
    force = LBMForce()
    force.setForceGroup(node.getIntProperty('forceGroup', 0))
    force.setName(node.getStringProperty('name', force.getName()))
    force.setGridSize(node.getIntProperty('nx'), node.getIntProperty('ny'), node.getIntProperty('nz'))
    force.setFluidDensity(node.getDoubleProperty('density'))
    force.setKinematicViscosity(node.getDoubleProperty('viscosity'))
    force.setFriction(node.getDoubleProperty('friction'))
    force.setTemperature(node.getDoubleProperty('temperature'))
    force.setRandomNumberSeed(node.getIntProperty('randomSeed'))
    force.setFluidMomentumRemovalFrequency(node.getIntProperty('momentumRemovalFrequency'))
    if version >= 2:
        force.setMachCheckFrequency(node.getIntProperty('machCheckFrequency'))
        force.setMachNumberLimit(node.getDoubleProperty('machNumberLimit'))
    if version >= 3:
        force.setCouplingScheme(node.getIntProperty('couplingScheme'))
    # Versions 1 to 3 predate the drag scheme (explicit drag), 1 to 8 the stencils (nearest node), 1 to 4 the
    # fluid fluctuations (none), 1 to 7 the domain decomposition (one domain), 1 to 5 the wall schemes
    # (bounce-back), 1 to 6 the open faces (a periodic box).
    if version >= 4:
        force.setDragScheme(node.getIntProperty('dragScheme'))
    if version >= 9:
        force.setInterpolationStencil(node.getIntProperty('interpolationStencil'))
    if version >= 5:
        force.setFluidFluctuations(node.getBoolProperty('fluidFluctuations'))
    if version >= 8:
        force.setDomainDecomposition(node.getIntProperty('domainsX'), node.getIntProperty('domainsY'),
                                     node.getIntProperty('domainsZ'))
        force.setParticleCopiesCheck(node.getBoolProperty('particleCopiesCheck', True))
        force.setDensityHaloExchange(node.getBoolProperty('densityHaloExchange', False))
        force.setVelocityHaloExchange(node.getBoolProperty('velocityHaloExchange', False))
    if version >= 6:
        force.setWallScheme(node.getIntProperty('wallScheme'))
    g = node.getChildNode('BodyAcceleration')
    force.setBodyAcceleration((g.getDoubleProperty('x'), g.getDoubleProperty('y'), g.getDoubleProperty('z')))
    u = node.getChildNode('InitialFluidVelocity')
    force.setInitialFluidVelocity((u.getDoubleProperty('x'), u.getDoubleProperty('y'), u.getDoubleProperty('z')))
    for particle in node.getChildNode('Particles').children:
        force.addParticle(particle.getIntProperty('index'))
    if version >= 2:
        force.setSolidNodes([solid.getIntProperty('index') for solid in node.getChildNode('SolidNodes').children])
    if version >= 7:
        faces = node.getChildNode('Faces').children
        if len(faces) != 6:
            raise SerializationError('LBMForce: the serialized force must have 6 faces')
        for face in range(6):
            force.setFaceBoundary(face, faces[face].getIntProperty('type'))
            force.setFaceVelocity(face, (faces[face].getDoubleProperty('vx'), faces[face].getDoubleProperty('vy'),
                                         faces[face].getDoubleProperty('vz')))
            force.setFaceDensity(face, faces[face].getDoubleProperty('density'))
    return force


def _encode(node, name, depth, lines):
    attributes = ''.join(' %s=%s' % (key, _quote(node.properties[key])) for key in sorted(node.properties))
    indent = '\t'*depth
    if not node.children:
        lines.append('%s<%s%s/>' % (indent, name, attributes))
        return
    lines.append('%s<%s%s>' % (indent, name, attributes))
    for child in node.children:
        _encode(child, child.name, depth + 1, lines)
    lines.append('%s</%s>' % (indent, name))


def _quote(value):
    return '"%s"' % escape(value, {'"': '&quot;'})


def _decode(element):
    node = SerializationNode(element.tag)
    node.properties = dict(element.attrib)
    node.children = [_decode(child) for child in element]
    return node


class XmlSerializer:
    """OpenMM's XmlSerializer for LBMForce."""

    @staticmethod
    def serialize(force, rootName='Force'):
        node = SerializationNode(rootName)
        node.setStringProperty('type', 'LBMForce')
        serialize_node(force, node)
        lines = ['<?xml version="1.0" ?>']
        _encode(node, rootName, 0, lines)
        return '\n'.join(lines) + '\n'

    @staticmethod
    def deserialize(text):
        try:
            root = ElementTree.fromstring(text.encode() if isinstance(text, str) else text)
        except ElementTree.ParseError as error:
            raise SerializationError('the XML could not be parsed: %s' % error)
        node = _decode(root)
        kind = node.getStringProperty('type', 'LBMForce')
        if kind != 'LBMForce':
            raise SerializationError("There is no serialization proxy registered for type %s" % kind)
        return deserialize_node(node)
