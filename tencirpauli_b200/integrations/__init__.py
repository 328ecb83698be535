"""Interoperability adapters for native MVP plans."""
