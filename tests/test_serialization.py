"""CPU tests of the XML serialization of LBMForce (lbm_b200.XmlSerializer), the reference's own test restated
(serialization/tests/TestSerializeLBMForce.cpp:22-197): a force with values different from the defaults survives
serialization, and the same document edited back to versions 8 to 3 (the attributes that those versions lacked
erased, the version number changed) reads with the settings of that time."""
import pytest

from lbm_b200 import LBMForce, XmlSerializer
from lbm_b200.serialization import SerializationError


def reference_force():
    force = LBMForce()
    force.setForceGroup(3)
    force.setName('fluid')
    force.setGridSize(10, 12, 14)
    force.setDomainDecomposition(2, 0, 3)
    force.setParticleCopiesCheck(False)
    force.setDensityHaloExchange(True)
    force.setVelocityHaloExchange(True)
    force.setFluidDensity(500.0)
    force.setKinematicViscosity(2.5)
    force.setFriction(5.0)
    force.setTemperature(310.0)
    force.setRandomNumberSeed(123)
    force.setFluidMomentumRemovalFrequency(10)
    force.setMachCheckFrequency(25)
    force.setMachNumberLimit(0.2)
    force.setCouplingScheme(LBMForce.NVE)
    force.setDragScheme(LBMForce.Centered)
    force.setInterpolationStencil(LBMForce.ThreePoint)
    force.setFluidFluctuations(True)
    force.setWallScheme(LBMForce.Regularized)
    force.setFaceBoundary(LBMForce.YMin, LBMForce.Density)
    force.setFaceBoundary(LBMForce.YMax, LBMForce.Velocity)
    force.setFaceDensity(LBMForce.YMin, 610.0)
    force.setFaceVelocity(LBMForce.YMax, (0.1, -0.2, 0.3))
    force.setFaceBoundary(LBMForce.ZMin, LBMForce.DensityVelocity)
    force.setFaceBoundary(LBMForce.ZMax, LBMForce.DensityVelocity)
    force.setFaceDensity(LBMForce.ZMin, 590.0)
    force.setFaceVelocity(LBMForce.ZMin, (-0.2, 0.1, 0.4))
    force.setSolidNodes([0, 7, 42])
    force.setBodyAcceleration((0.1, 0.2, 0.3))
    force.setInitialFluidVelocity((-0.1, 0.0, 0.05))
    force.addParticle(3)
    force.addParticle(7)
    force.addParticle(1)
    return force


GETTERS = ['getForceGroup', 'getName', 'getGridSize', 'getDomainDecomposition', 'getParticleCopiesCheck',
           'getDensityHaloExchange', 'getVelocityHaloExchange', 'getFluidDensity', 'getKinematicViscosity',
           'getFriction', 'getTemperature', 'getRandomNumberSeed', 'getFluidMomentumRemovalFrequency',
           'getMachCheckFrequency', 'getMachNumberLimit', 'getCouplingScheme', 'getDragScheme',
           'getInterpolationStencil', 'getFluidFluctuations', 'getWallScheme', 'getSolidNodes', 'getBodyAcceleration',
           'getInitialFluidVelocity', 'getNumParticles']


def test_round_trip():
    force = reference_force()
    copy = XmlSerializer.deserialize(XmlSerializer.serialize(force))
    for getter in GETTERS:
        assert getattr(copy, getter)() == getattr(force, getter)(), getter
    for face in range(6):
        assert copy.getFaceBoundary(face) == force.getFaceBoundary(face)
        assert copy.getFaceVelocity(face) == force.getFaceVelocity(face)
        assert copy.getFaceDensity(face) == force.getFaceDensity(face)
    assert [copy.getParticle(i) for i in range(3)] == [3, 7, 1]


def test_document_layout():
    xml = XmlSerializer.serialize(reference_force())
    lines = xml.splitlines()
    assert lines[0] == '<?xml version="1.0" ?>'
    assert lines[1].startswith('<Force ') and lines[-1] == '</Force>'
    for attribute in (' type="LBMForce"', ' version="9"', ' name="fluid"', ' interpolationStencil="2"',
                      ' fluidFluctuations="1"', ' wallScheme="1"', ' dragScheme="1"', ' domainsY="0"'):
        assert attribute in lines[1], attribute
    assert lines[2] == '\t<BodyAcceleration x="0.1" y="0.2" z="0.3"/>'
    assert '\t\t<Particle index="7"/>' in lines
    assert sum(line.startswith('\t\t<Face ') for line in lines) == 6


def edit(xml, erase=None, version=None):
    if erase is not None:
        assert erase in xml
        xml = xml.replace(erase, '', 1)
    if version is not None:
        old, new = 'version="%d"' % (version + 1), 'version="%d"' % version
        assert old in xml
        xml = xml.replace(old, new, 1)
    return xml


def test_older_versions():
    force = reference_force()
    xml = XmlSerializer.serialize(force)
    # Version 8 predates the interpolation stencils: the nearest node.
    xml = edit(xml, ' interpolationStencil="2"', 8)
    copy = XmlSerializer.deserialize(xml)
    assert copy.getInterpolationStencil() == LBMForce.NearestNode
    assert copy.getDragScheme() == LBMForce.Centered
    # Version 7 predates the domain decomposition: one domain, the copies checked, no halo exchange.
    xml = edit(xml, version=7)
    copy = XmlSerializer.deserialize(xml)
    assert copy.getDomainDecomposition() == (1, 1, 1)
    assert copy.getParticleCopiesCheck() and not copy.getDensityHaloExchange() and not copy.getVelocityHaloExchange()
    # Version 6 predates the open faces: a periodic box (the wall scheme is still read).
    xml = edit(xml, version=6)
    copy = XmlSerializer.deserialize(xml)
    assert all(copy.getFaceBoundary(face) == LBMForce.Periodic for face in range(6))
    assert copy.getWallScheme() == LBMForce.Regularized
    # Version 5 predates the wall schemes: bounce-back.
    xml = edit(xml, ' wallScheme="1"', 5)
    copy = XmlSerializer.deserialize(xml)
    assert copy.getWallScheme() == LBMForce.BounceBack and copy.getFluidFluctuations()
    # Version 4 predates the fluid fluctuations: none.
    xml = edit(xml, ' fluidFluctuations="1"', 4)
    copy = XmlSerializer.deserialize(xml)
    assert not copy.getFluidFluctuations() and copy.getDragScheme() == LBMForce.Centered
    # Version 3 predates the drag scheme: the explicit drag.
    xml = edit(xml, ' dragScheme="1"', 3)
    copy = XmlSerializer.deserialize(xml)
    assert copy.getDragScheme() == LBMForce.Explicit and not copy.getFluidFluctuations()
    assert copy.getCouplingScheme() == force.getCouplingScheme()


def test_errors():
    xml = XmlSerializer.serialize(reference_force())
    with pytest.raises(SerializationError, match='Unsupported version number'):
        XmlSerializer.deserialize(xml.replace('version="9"', 'version="10"'))
    with pytest.raises(SerializationError, match="Unknown property 'nx'"):
        XmlSerializer.deserialize(xml.replace(' nx="10"', ''))
    start = xml.index('\t\t<Face ')
    with pytest.raises(SerializationError, match='must have 6 faces'):
        XmlSerializer.deserialize(xml[:start] + xml[xml.index('\n', start) + 1:])
    with pytest.raises(SerializationError, match='no serialization proxy'):
        XmlSerializer.deserialize(xml.replace('type="LBMForce"', 'type="HarmonicBondForce"'))


def test_a_context_rejects_more_than_one_domain():
    force = reference_force()
    with pytest.raises(ValueError, match='more than one domain'):
        force.latticeParameters([10.0, 12.0, 14.0], 0.01, [1.0]*8)
