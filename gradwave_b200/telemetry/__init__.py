"""Telemetry hooks of the band-solve path."""
