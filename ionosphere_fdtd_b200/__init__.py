"""B200-native engine for the geodesic FDTD time step of ionosphere-fdtd.

Public names follow the reference package (``ionosphere_fdtd``) so that code
written against its PyTorch CUDA backend switches by changing the import.
"""

from .adaptive_mesh import (
    AdaptiveMeshValidation,
    SphericalRefinementRegion,
    build_adaptive_geodesic_mesh,
    validate_adaptive_mesh,
)
from .backend import ArrayBackend, CudaBackend, TorchBackend, create_backend
from .checkpoint import load_checkpoint, save_checkpoint
from .constants import C_0, EARTH_RADIUS_M, EPSILON_0, MU_0
from .ensemble import Ensemble
from .errors import BackendUnavailableError, CheckpointError
from .materials import EarthIonosphereMaterial, SphericalAnomaly
from .mesh import (
    GeodesicMesh,
    build_geodesic_mesh,
    build_geodesic_mesh_from_topology,
    build_geodesic_mesh_from_vertices,
)
from .plasma import (
    ELECTRON_MASS_KG,
    ELEMENTARY_CHARGE_C,
    ColdPlasmaSpecies,
    GeodesicPlasmaCoupler,
    MagnetizedPlasmaADE,
    MeshPlasmaModel,
)
from .provenance import DataArtifactError, DatasetProvenance, VariableProvenance, array_sha256
from .radial_grid import RadialGridValidation, RadialRefinementRegion, build_refined_radial_grid, validate_radial_grid
from .receivers import Receiver, ReceiverTraces, receiver_location, record_receiver_traces
from .solver import GeodesicFDTD, SimulationConfig
from .sources import (
    GaussianCurrent,
    TangentialGaussianCurrent,
    geographic_direction,
    geographic_distribution,
    geographic_face_index,
    radial_linear_distribution,
)
from .surface_impedance import ConductiveHalfSpaceSurface, SurfaceImpedanceADE

__version__ = "0.1.0"

__all__ = [
    "AdaptiveMeshValidation",
    "SphericalRefinementRegion",
    "build_adaptive_geodesic_mesh",
    "validate_adaptive_mesh",
    "Ensemble",
    "ArrayBackend",
    "TorchBackend",
    "DataArtifactError",
    "BackendUnavailableError",
    "C_0",
    "CheckpointError",
    "ColdPlasmaSpecies",
    "ConductiveHalfSpaceSurface",
    "CudaBackend",
    "DatasetProvenance",
    "EARTH_RADIUS_M",
    "ELECTRON_MASS_KG",
    "ELEMENTARY_CHARGE_C",
    "EPSILON_0",
    "EarthIonosphereMaterial",
    "GaussianCurrent",
    "GeodesicFDTD",
    "GeodesicMesh",
    "GeodesicPlasmaCoupler",
    "MU_0",
    "MagnetizedPlasmaADE",
    "MeshPlasmaModel",
    "SimulationConfig",
    "SphericalAnomaly",
    "SurfaceImpedanceADE",
    "TangentialGaussianCurrent",
    "VariableProvenance",
    "array_sha256",
    "build_geodesic_mesh",
    "build_geodesic_mesh_from_topology",
    "build_geodesic_mesh_from_vertices",
    "create_backend",
    "geographic_direction",
    "geographic_distribution",
    "geographic_face_index",
    "load_checkpoint",
    "radial_linear_distribution",
    "RadialGridValidation",
    "RadialRefinementRegion",
    "build_refined_radial_grid",
    "validate_radial_grid",
    "Receiver",
    "ReceiverTraces",
    "receiver_location",
    "record_receiver_traces",
    "save_checkpoint",
]
