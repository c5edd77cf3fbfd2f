"""Version of the fresnel API this package mirrors (fresnel/version.py:10) and of the engine."""

version = "0.13.5"
engine_version = "0.1.0"
