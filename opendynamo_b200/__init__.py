"""opendynamo-b200: a B200-native (sm_100a) FR P=3 compressible Navier-Stokes
step path behind the surface of OpenDynamo (config.toml schema, state files,
labels, checkpoint/resume, flux / wall / precision choices)."""

__version__ = "0.1.0"
