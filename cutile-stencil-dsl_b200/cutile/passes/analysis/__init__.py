"""Footprint and roofline analysis passes."""
